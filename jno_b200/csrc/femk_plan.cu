// Plan build on the device: P2 numbering, DOF -> element incidence, the compress-plan CSR
// pattern, the element -> slot map, diagonal slots and the boundary-facet Dirichlet set.
//
// Reference behaviour reproduced (pinned by the oracle tests):
//  * P2 DOFs: vertices keep ids 0..nv-1, edge midpoints are numbered in first-encounter order over
//    (cell, local dof), local edge order (2,3),(1,3),(1,2),(0,3),(0,2),(0,1)
//    (jno/utils/solver/fem_utils.py:1979-2044, jno/utils/solver/fem_topology.py:44).
//  * Pattern: the unique (row, col) pairs of all element dofs, rows ascending, columns ascending
//    within a row (compress_plan, fem_utils.py:4049-4057); slot[c, a, b] is the plan's inverse.
//  * Dirichlet: every node on a facet owned by exactly one tet (jno/_fem.py:2695).
//
// Everything here is integer work: one thread (or warp) per element/row, no sorting library.
#include <algorithm>
#include <atomic>
#include <climits>
#include <thread>
#include <vector>

#include "femk_element.cuh"
#include "femk_internal.cuh"
#include "femk_spmv.cuh"

namespace femk {
namespace {

// Simplex topology: NV vertices, NE = NV (NV - 1) / 2 edges in basix order (cell_edge_a/b), and
// NV facets, facet f being the NV - 1 vertices other than f (the facet set of a tetrahedron /
// triangle; only the set matters to the boundary test).
template <int NV>
__host__ __device__ constexpr int n_edges() {
  return NV * (NV - 1) / 2;
}
// local edge index of the vertex pair (i, j), i != j
template <int NV>
__device__ __forceinline__ int local_edge(int i, int j) {
  int found = 0;
#pragma unroll
  for (int e = 0; e < n_edges<NV>(); ++e) {
    const int a = cell_edge_a<NV>(e), b = cell_edge_b<NV>(e);
    if ((a == i && b == j) || (a == j && b == i)) found = e;
  }
  return found;
}

constexpr int kThreads = 256;

__global__ void k_count(const int32_t* __restrict__ cells, int64_t m, int64_t n,
                        unsigned long long* __restrict__ cnt, int* __restrict__ err) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < m; t += (int64_t)gridDim.x * blockDim.x) {
    const int32_t v = cells[t];
    if (v < 0 || v >= n) {
      atomicOr(err, 1);
      continue;
    }
    atomicAdd(&cnt[v], 1ull);
  }
}

// Connectivity check before any kernel indexes with it: every id in [0, nvert) and the NV
// vertices of an element pairwise distinct. Reads the cells only; writes the error flag.
template <int NV>
__global__ void k_validate_cells(const int32_t* __restrict__ tets, int64_t ntet, int64_t nvert,
                                 int* __restrict__ err) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ntet; c += (int64_t)gridDim.x * blockDim.x) {
    int32_t v[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = tets[c * NV + q];
    bool bad = false;
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      bad |= v[q] < 0 || v[q] >= nvert;
#pragma unroll
      for (int r = q + 1; r < NV; ++r) bad |= v[q] == v[r];
    }
    if (bad) atomicOr(err, 1);
  }
}

__global__ void k_to_i32(const int64_t* __restrict__ in, int64_t n, int32_t* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (int32_t)in[i];
}

template <int ND>
__global__ void k_fill(const int32_t* __restrict__ cells, int64_t ntet, int64_t n, const int32_t* __restrict__ ptr,
                       int32_t* __restrict__ cursor, int32_t* __restrict__ inc) {
  const int64_t m = ntet * ND;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < m; t += (int64_t)gridDim.x * blockDim.x) {
    const int32_t v = cells[t];
    if (v < 0 || v >= n) continue;  // rejected earlier by k_validate_tets / k_count
    const int32_t pos = atomicAdd(&cursor[v], 1);
    inc[ptr[v] + pos] = (int32_t)(t / ND);
  }
}

// Sort each incidence list ascending (lists are short: the element valence of a node).
__global__ void k_sort_lists(const int32_t* __restrict__ ptr, int64_t n, int32_t* __restrict__ inc) {
  for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
    const int32_t b = ptr[v], e = ptr[v + 1];
    for (int32_t i = b + 1; i < e; ++i) {
      const int32_t key = inc[i];
      int32_t j = i - 1;
      while (j >= b && inc[j] > key) {
        inc[j + 1] = inc[j];
        --j;
      }
      inc[j + 1] = key;
    }
  }
}

// For every (cell, local edge): the raw index c'*NE+e' of the first cell containing the same edge.
template <int NV>
__global__ void k_edge_first(const int32_t* __restrict__ tets, int64_t ntet, const int32_t* __restrict__ vptr,
                             const int32_t* __restrict__ vinc, int32_t* __restrict__ first_raw,
                             int64_t* __restrict__ is_first, int* __restrict__ err) {
  constexpr int NE = n_edges<NV>();
  const int64_t m = ntet * NE;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < m; r += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = r / NE;
    const int e = (int)(r % NE);
    const int32_t a = tets[c * NV + cell_edge_a<NV>(e)], b = tets[c * NV + cell_edge_b<NV>(e)];
    const int32_t u = min(a, b), w = max(a, b);
    int64_t found = -1;
    for (int32_t j = vptr[u]; j < vptr[u + 1] && found < 0; ++j) {
      const int32_t c2 = vinc[j];
      int iu = -1, iw = -1;
#pragma unroll
      for (int q = 0; q < NV; ++q) {
        const int32_t t = tets[(int64_t)c2 * NV + q];
        if (t == u) iu = q;
        if (t == w) iw = q;
      }
      if (iw >= 0 && iu >= 0) found = (int64_t)c2 * NE + local_edge<NV>(iu, iw);
    }
    if (found < 0) {
      atomicOr(err, 2);
      found = r;
    }
    first_raw[r] = (int32_t)found;
    is_first[r] = found == r ? 1 : 0;
  }
}

// P2 connectivity (vertices, then the edge midpoints numbered by first encounter) and midpoint
// coordinates; xyz and points hold 3 coordinates per node.
template <int NV>
__global__ void k_p2_cells(const int32_t* __restrict__ tets, int64_t ntet, int64_t nvert,
                           const int32_t* __restrict__ first_raw, const int64_t* __restrict__ rank,
                           const double* __restrict__ xyz, int32_t* __restrict__ cells, double* __restrict__ points) {
  constexpr int NE = n_edges<NV>(), ND = NV + NE;
  const int64_t m = ntet * NE;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < m; r += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = r / NE;
    const int e = (int)(r % NE);
    const int64_t fr = first_raw[r];
    const int64_t id = nvert + rank[fr];
    cells[c * ND + NV + e] = (int32_t)id;
    if (e < NV) cells[c * ND + e] = tets[c * NV + e];  // NE >= NV
    if (fr == r) {
      const int32_t a = tets[c * NV + cell_edge_a<NV>(e)], b = tets[c * NV + cell_edge_b<NV>(e)];
#pragma unroll
      for (int k = 0; k < 3; ++k) points[id * 3 + k] = 0.5 * xyz[(int64_t)a * 3 + k] + 0.5 * xyz[(int64_t)b * 3 + k];
    }
  }
}

__device__ __forceinline__ int warp_min_i32(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Row pattern by repeated warp-wide minimum extraction over the candidate dofs of a row's
// incident elements: no sort, deterministic, each row's columns ascending.
template <int ND>
__global__ void k_row_pattern(const int32_t* __restrict__ cells, const int32_t* __restrict__ inc_ptr,
                              const int32_t* __restrict__ inc, int64_t n, const int64_t* __restrict__ rowptr,
                              int64_t* __restrict__ rowlen, int32_t* __restrict__ cols, int* __restrict__ max_len) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t row = warp; row < n; row += nwarps) {
    const int32_t beg = inc_ptr[row];
    const int32_t m = (inc_ptr[row + 1] - beg) * ND;
    int prev = -1;
    int32_t count = 0;
    const int64_t out = cols ? rowptr[row] : 0;
    while (true) {
      int best = INT_MAX;
      for (int32_t idx = lane; idx < m; idx += 32) {
        const int32_t c = inc[beg + idx / ND];
        const int v = cells[(int64_t)c * ND + idx % ND];
        if (v > prev && v < best) best = v;
      }
      best = warp_min_i32(best);
      if (best == INT_MAX) break;
      if (cols && lane == 0) cols[out + count] = best;
      ++count;
      prev = best;
    }
    if (lane == 0) {
      rowlen[row] = count;
      atomicMax(max_len, count);
    }
  }
}

__device__ __forceinline__ int32_t find_col(const int32_t* __restrict__ cols, int32_t lo, int32_t hi, int32_t key) {
  while (lo < hi) {
    const int32_t mid = (lo + hi) >> 1;
    if (cols[mid] < key)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

template <int ND>
__global__ void k_slot_map(const int32_t* __restrict__ cells, int64_t ntet, const int32_t* __restrict__ indptr,
                           const int32_t* __restrict__ indices, int32_t* __restrict__ slot, int* __restrict__ err) {
  const int64_t m = ntet * ND;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < m; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = t / ND;
    const int32_t row = cells[t];
    const int32_t lo = indptr[row], hi = indptr[row + 1];
#pragma unroll
    for (int b = 0; b < ND; ++b) {
      const int32_t col = cells[c * ND + b];
      const int32_t pos = find_col(indices, lo, hi, col);
      if (pos >= hi || indices[pos] != col) atomicOr(err, 4);
      slot[t * ND + b] = pos;
    }
  }
}

__global__ void k_diag_slot(const int32_t* __restrict__ indptr, const int32_t* __restrict__ indices, int64_t n,
                            int32_t* __restrict__ diag, int* __restrict__ err) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t lo = indptr[i], hi = indptr[i + 1];
    const int32_t pos = find_col(indices, lo, hi, (int32_t)i);
    if (pos >= hi || indices[pos] != i) atomicOr(err, 8);
    diag[i] = pos;
  }
}

// A facet (the NV - 1 vertices other than vertex f) is on the boundary when no other element has
// all of its vertices; P2 marks the midpoints of the facet's edges too.
template <int ND>
__global__ void k_boundary(const int32_t* __restrict__ cells, int64_t ntet, const int32_t* __restrict__ vptr,
                           const int32_t* __restrict__ vinc, uint8_t* __restrict__ mask) {
  constexpr int NV = Cell<ND>::NV;
  const int64_t m = ntet * NV;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < m; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = t / NV;
    const int f = (int)(t % NV);
    int32_t v[NV - 1];
    int32_t lo = INT_MAX;
#pragma unroll
    for (int q = 0, k = 0; q < NV; ++q)
      if (q != f) {
        v[k] = cells[c * ND + q];
        lo = min(lo, v[k]);
        ++k;
      }
    bool shared = false;
    for (int32_t j = vptr[lo]; j < vptr[lo + 1] && !shared; ++j) {
      const int32_t c2 = vinc[j];
      if (c2 == c) continue;
      int hit = 0;
#pragma unroll
      for (int q = 0; q < NV; ++q) {
        const int32_t w = cells[(int64_t)c2 * ND + q];
#pragma unroll
        for (int k = 0; k < NV - 1; ++k) hit += w == v[k];
      }
      shared = hit == NV - 1;
    }
    if (shared) continue;
#pragma unroll
    for (int k = 0; k < NV - 1; ++k) mask[v[k]] = 1;
    if (Cell<ND>::P2) {
#pragma unroll
      for (int e = 0; e < n_edges<NV>(); ++e)
        if (cell_edge_a<NV>(e) != f && cell_edge_b<NV>(e) != f) mask[cells[c * ND + NV + e]] = 1;
    }
  }
}

__global__ void k_mask_to_i64(const uint8_t* __restrict__ mask, int64_t n, int64_t* __restrict__ flag) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    flag[i] = mask[i] ? 1 : 0;
}

__global__ void k_compact(const uint8_t* __restrict__ mask, const int64_t* __restrict__ pos, int64_t n,
                          int32_t* __restrict__ list) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    if (mask[i]) list[pos[i]] = (int32_t)i;
}

// Largest CSR span of R consecutive rows (one value per block of the row-gather assembly).
__global__ void k_block_span(const int32_t* __restrict__ indptr, int64_t n, int R, int64_t nblk,
                             unsigned long long* __restrict__ out) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nblk; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r0 = t * R, r1 = r0 + R < n ? r0 + R : n;
    atomicMax(out, (unsigned long long)(indptr[r1] - indptr[r0]));
  }
}

// Width of each 32-row slice (its longest row) and its entry count.
__global__ void k_sell_width(const int32_t* __restrict__ indptr, int64_t n, int64_t nslices, int64_t* __restrict__ len) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t sl = warp; sl < nslices; sl += nwarps) {
    const int64_t row = sl * 32 + lane;
    int w = row < n ? indptr[row + 1] - indptr[row] : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) w = max(w, __shfl_xor_sync(0xffffffffu, w, o));
    if (lane == 0) len[sl] = (int64_t)w * 32;
  }
}

__global__ void k_sell_fill(const int32_t* __restrict__ indptr, const int32_t* __restrict__ indices, int64_t n,
                            int64_t nslices, const int64_t* __restrict__ sptr, int32_t* __restrict__ cols,
                            int16_t* __restrict__ c16) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t sl = warp; sl < nslices; sl += nwarps) {
    const int64_t row = sl * 32 + lane;
    const int64_t w = (sptr[sl + 1] - sptr[sl]) / 32;
    const int32_t beg = row < n ? indptr[row] : 0;
    const int32_t len = row < n ? indptr[row + 1] - beg : 0;
    const int64_t self = row < n ? row : n - 1;
    for (int64_t k = 0; k < w; ++k) {
      const int64_t j = sptr[sl] + k * 32 + lane;
      const bool real = k < len;
      const int32_t col = real ? indices[beg + k] : (int32_t)self;
      cols[j] = col;
      if (c16) c16[j] = (int16_t)(col - self);
    }
  }
}

__global__ void k_cols16(const int32_t* __restrict__ indptr, const int32_t* __restrict__ indices, int64_t n,
                         int16_t* __restrict__ c16, int* __restrict__ bad) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    for (int32_t k = indptr[i]; k < indptr[i + 1]; ++k) {
      const int64_t d = (int64_t)indices[k] - i;
      if (d < -32768 || d > 32767) {
        atomicOr(bad, 1);
        c16[k] = 0;
      } else {
        c16[k] = (int16_t)d;
      }
    }
  }
}

// coordinates with dim components per vertex -> 3 per vertex (z = 0 in 2-D) in a (and b)
__global__ void k_copy_xyz(const double* __restrict__ in, int64_t nvert, int dim, double* __restrict__ a,
                           double* __restrict__ b) {
  const int64_t m = nvert * 3;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t v = i / 3;
    const int k = (int)(i % 3);
    const double x = k < dim ? in[v * dim + k] : 0.0;
    a[i] = x;
    if (b) b[i] = x;
  }
}

template <typename T>
int dev_alloc(T** p, int64_t count, cudaStream_t s) {
  if (count <= 0) count = 1;
  FEMK_CUDA_TRY(cudaMalloc((void**)p, sizeof(T) * count));
  (void)s;
  return FEMK_OK;
}

struct Temp {
  void* p = nullptr;
  ~Temp() {
    if (p) cudaFree(p);
  }
};

int read_err(int* d_err, cudaStream_t s, int* h) {
  FEMK_CUDA_TRY(cudaMemcpyAsync(h, d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
  FEMK_CUDA_TRY(cudaStreamSynchronize(s));
  return FEMK_OK;
}

// incidence of `cells` (nd per element) over n dofs into plan-owned ptr/inc arrays
template <int ND>
int build_incidence(const int32_t* cells, int64_t ntet, int64_t n, int32_t** ptr_out, int32_t** inc_out,
                    int* d_err, cudaStream_t s) {
  Temp cnt, scan, cur;
  FEMK_CUDA_TRY(cudaMalloc(&cnt.p, sizeof(int64_t) * (n + 1)));
  FEMK_CUDA_TRY(cudaMalloc(&scan.p, sizeof(int64_t) * (n + 1)));
  FEMK_CUDA_TRY(cudaMemsetAsync(cnt.p, 0, sizeof(int64_t) * (n + 1), s));
  const int64_t m = ntet * ND;
  k_count<<<::femk::counted_launch() + blocks_for(m, kThreads, 65535 * 4), kThreads, 0, s>>>(cells, m, n, (unsigned long long*)cnt.p, d_err);
  FEMK_CUDA_TRY(cudaGetLastError());
  int h_err = 0;
  FEMK_TRY(read_err(d_err, s, &h_err));
  if (h_err) {
    set_error("femk_plan_create: connectivity references a DOF outside [0, n)");
    return FEMK_EINVAL;
  }
  FEMK_TRY(scan_exclusive_i64((const int64_t*)cnt.p, (int64_t*)scan.p, n, s));
  FEMK_TRY(dev_alloc(ptr_out, n + 1, s));
  FEMK_TRY(dev_alloc(inc_out, m, s));
  k_to_i32<<<::femk::counted_launch() + blocks_for(n + 1, kThreads, 65535 * 4), kThreads, 0, s>>>((const int64_t*)scan.p, n + 1, *ptr_out);
  FEMK_CUDA_TRY(cudaMalloc(&cur.p, sizeof(int32_t) * (n + 1)));
  FEMK_CUDA_TRY(cudaMemsetAsync(cur.p, 0, sizeof(int32_t) * (n + 1), s));
  k_fill<ND><<<::femk::counted_launch() + blocks_for(m, kThreads, 65535 * 4), kThreads, 0, s>>>(cells, ntet, n, *ptr_out, (int32_t*)cur.p, *inc_out);
  k_sort_lists<<<::femk::counted_launch() + blocks_for(n, 128, 65535 * 4), 128, 0, s>>>(*ptr_out, n, *inc_out);
  FEMK_CUDA_TRY(cudaGetLastError());
  FEMK_CUDA_TRY(cudaStreamSynchronize(s));  // temporaries are freed on return
  return FEMK_OK;
}

int build_uniform_columns(femk_plan* p, cudaStream_t s);

template <int ND>
int build_pattern(femk_plan* p, int* d_err, int* h_err, cudaStream_t s) {
  const int64_t n = p->n;
  Temp rowlen, rowptr, dmax;
  FEMK_CUDA_TRY(cudaMalloc(&rowlen.p, sizeof(int64_t) * (n + 1)));
  FEMK_CUDA_TRY(cudaMalloc(&rowptr.p, sizeof(int64_t) * (n + 1)));
  FEMK_CUDA_TRY(cudaMalloc(&dmax.p, sizeof(int)));
  FEMK_CUDA_TRY(cudaMemsetAsync(dmax.p, 0, sizeof(int), s));
  const int warps_blocks = blocks_for(n * 32, kThreads, p->n_sm * 64);
  k_row_pattern<ND><<<::femk::counted_launch() + warps_blocks, kThreads, 0, s>>>(p->cells, p->inc_ptr, p->inc_elem, n, nullptr,
                                                      (int64_t*)rowlen.p, nullptr, (int*)dmax.p);
  FEMK_CUDA_TRY(cudaGetLastError());
  FEMK_TRY(scan_exclusive_i64((const int64_t*)rowlen.p, (int64_t*)rowptr.p, n, s));
  int64_t nnz = 0;
  FEMK_CUDA_TRY(cudaMemcpyAsync(&nnz, (int64_t*)rowptr.p + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  FEMK_CUDA_TRY(cudaMemcpyAsync(&p->max_row, dmax.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  FEMK_CUDA_TRY(cudaStreamSynchronize(s));
  if (nnz >= INT32_MAX) {
    set_error("femk_plan_create: the CSR pattern has >= 2^31 entries; int32 indptr cannot hold it");
    return FEMK_EINVAL;
  }
  p->nnz = nnz;
  if (p->spmv_L == 0) choose_spmv_cfg(n > 0 ? (double)nnz / (double)n : 1.0, &p->spmv_L, &p->spmv_U);
  FEMK_TRY(dev_alloc(&p->indptr, n + 1, s));
  FEMK_TRY(dev_alloc(&p->indices, nnz, s));
  k_to_i32<<<::femk::counted_launch() + blocks_for(n + 1, kThreads, 65535 * 4), kThreads, 0, s>>>((const int64_t*)rowptr.p, n + 1, p->indptr);
  k_row_pattern<ND><<<::femk::counted_launch() + warps_blocks, kThreads, 0, s>>>(p->cells, p->inc_ptr, p->inc_elem, n, (const int64_t*)rowptr.p,
                                                      (int64_t*)rowlen.p, p->indices, (int*)dmax.p);
  FEMK_TRY(dev_alloc(&p->slot, p->ntet * ND * ND, s));
  k_slot_map<ND><<<::femk::counted_launch() + blocks_for(p->ntet * ND, kThreads, 65535 * 4), kThreads, 0, s>>>(p->cells, p->ntet, p->indptr,
                                                                                    p->indices, p->slot, d_err);
  // rows per block of the row-gather assembly: as many as keep the block's staged span (8 B value +
  // 4 B column per entry) within 64 KB of shared memory
  {
    Temp span;
    FEMK_CUDA_TRY(cudaMalloc(&span.p, sizeof(unsigned long long)));
    int R = ND <= 4 ? 128 : 64;
    while (true) {
      FEMK_CUDA_TRY(cudaMemsetAsync(span.p, 0, sizeof(unsigned long long), s));
      const int64_t nblk = (n + R - 1) / R;
      k_block_span<<<::femk::counted_launch() + blocks_for(nblk, kThreads, 65535 * 4), kThreads, 0, s>>>(
          p->indptr, n, R, nblk, (unsigned long long*)span.p);
      unsigned long long h = 0;
      FEMK_CUDA_TRY(cudaMemcpyAsync(&h, span.p, sizeof(h), cudaMemcpyDeviceToHost, s));
      FEMK_CUDA_TRY(cudaStreamSynchronize(s));
      if (h * 12 <= 65536 || R == 32) {
        p->asm_rows = R;
        p->asm_span = (int64_t)h;
        break;
      }
      R /= 2;
    }
    if (p->asm_span * 12 > 200 * 1024) {
      set_error("femk_plan_create: rows too long for the shared-memory assembly");
      return FEMK_EINVAL;
    }
  }
  FEMK_TRY(dev_alloc(&p->diag, n, s));
  k_diag_slot<<<::femk::counted_launch() + blocks_for(n, kThreads, 65535 * 4), kThreads, 0, s>>>(p->indptr, p->indices, n, p->diag, d_err);
  FEMK_CUDA_TRY(cudaGetLastError());
  FEMK_TRY(read_err(d_err, s, h_err));
  if (*h_err) {
    set_error("femk_plan_create: slot map or diagonal lookup failed (corrupt connectivity?)");
    return FEMK_EBOUNDS;
  }
  // compact int16 column offsets for the FP32 inner solve
  int* d_bad = nullptr;
  FEMK_CUDA_TRY(cudaMalloc(&d_bad, sizeof(int)));
  Temp bad;
  bad.p = d_bad;
  FEMK_CUDA_TRY(cudaMemsetAsync(d_bad, 0, sizeof(int), s));
  FEMK_TRY(dev_alloc(&p->cols16, nnz, s));
  k_cols16<<<::femk::counted_launch() + blocks_for(n, kThreads, 65535 * 4), kThreads, 0, s>>>(p->indptr, p->indices, n, p->cols16, d_bad);
  int hbad = 0;
  FEMK_TRY(read_err(d_bad, s, &hbad));
  if (hbad) {
    cudaFree(p->cols16);
    p->cols16 = nullptr;
  }
  // sliced-ELL copy of the pattern for the solver
  p->n_slices = (n + 31) / 32;
  Temp slen;
  FEMK_CUDA_TRY(cudaMalloc(&slen.p, sizeof(int64_t) * (p->n_slices + 1)));
  FEMK_TRY(dev_alloc(&p->sell_ptr, p->n_slices + 1, s));
  const int sgrid = blocks_for(p->n_slices * 32, kThreads, p->n_sm * 64);
  k_sell_width<<<::femk::counted_launch() + sgrid, kThreads, 0, s>>>(p->indptr, n, p->n_slices, (int64_t*)slen.p);
  FEMK_TRY(scan_exclusive_i64((const int64_t*)slen.p, p->sell_ptr, p->n_slices, s));
  FEMK_CUDA_TRY(cudaMemcpyAsync(&p->sell_nnz, p->sell_ptr + p->n_slices, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  FEMK_CUDA_TRY(cudaStreamSynchronize(s));
  if (p->sell_nnz >= INT32_MAX) {
    p->use_sell = 0;
    return FEMK_OK;
  }
  FEMK_TRY(dev_alloc(&p->sell_cols, p->sell_nnz, s));
  if (p->cols16) FEMK_TRY(dev_alloc(&p->sell_c16, p->sell_nnz, s));
  k_sell_fill<<<::femk::counted_launch() + sgrid, kThreads, 0, s>>>(p->indptr, p->indices, n, p->n_slices, p->sell_ptr,
                                                                    p->sell_cols, p->sell_c16);
  FEMK_CUDA_TRY(cudaGetLastError());
  FEMK_CUDA_TRY(cudaStreamSynchronize(s));
  return build_uniform_columns(p, s);
}

// Per-slice column table of the bulk-copy SpMV: a slice whose 32 rows share one column-offset
// sequence (every row of an interior stretch of a structured mesh line) stores it once
// (w offsets, padded to 8 = 16 bytes); any other slice keeps its 32*w per-entry offsets.
// len[s] = entries of slice s's table; the table of slice s starts at cptr[s] (a multiple of 8).
__global__ void k_sell_uni_len(const int64_t* __restrict__ sptr, const int16_t* __restrict__ c16, int64_t nslices,
                               int64_t* __restrict__ len) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t sl = warp; sl < nslices; sl += nwarps) {
    const int64_t b0 = sptr[sl];
    const int64_t w = (sptr[sl + 1] - b0) / 32;
    bool uni = true;
    for (int64_t k = 0; k < w && uni; ++k) {
      const int16_t c = c16[b0 + 32 * k + lane];
      uni = __all_sync(0xffffffffu, c == __shfl_sync(0xffffffffu, c, 0));
    }
    if (lane == 0) len[sl] = uni ? (w + 7) / 8 * 8 : 32 * w;
  }
}

__global__ void k_sell_uni_fill(const int64_t* __restrict__ sptr, const int16_t* __restrict__ c16, int64_t nslices,
                                const int64_t* __restrict__ cptr, int16_t* __restrict__ cu) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t sl = warp; sl < nslices; sl += nwarps) {
    const int64_t b0 = sptr[sl];
    const int64_t w = (sptr[sl + 1] - b0) / 32;
    const int64_t c0 = cptr[sl], len = cptr[sl + 1] - c0;
    if (len == 32 * w) {
      for (int64_t j = lane; j < len; j += 32) cu[c0 + j] = c16[b0 + j];
    } else {
      for (int64_t k = lane; k < len; k += 32) cu[c0 + k] = k < w ? c16[b0 + 32 * k] : (int16_t)0;
    }
  }
}

int build_uniform_columns(femk_plan* p, cudaStream_t s) {
  if (!p->sell_c16 || !p->sell_uni) return FEMK_OK;
  Temp len;
  FEMK_CUDA_TRY(cudaMalloc(&len.p, sizeof(int64_t) * (p->n_slices + 1)));
  FEMK_TRY(dev_alloc(&p->sell_cuptr, p->n_slices + 1, s));
  const int sgrid = blocks_for(p->n_slices * 32, kThreads, p->n_sm * 64);
  k_sell_uni_len<<<::femk::counted_launch() + sgrid, kThreads, 0, s>>>(p->sell_ptr, p->sell_c16, p->n_slices,
                                                                       (int64_t*)len.p);
  FEMK_TRY(scan_exclusive_i64((const int64_t*)len.p, p->sell_cuptr, p->n_slices, s));
  FEMK_CUDA_TRY(cudaMemcpyAsync(&p->sell_cu_len, p->sell_cuptr + p->n_slices, sizeof(int64_t), cudaMemcpyDeviceToHost,
                                s));
  FEMK_CUDA_TRY(cudaStreamSynchronize(s));
  FEMK_TRY(dev_alloc(&p->sell_cu, p->sell_cu_len, s));
  k_sell_uni_fill<<<::femk::counted_launch() + sgrid, kThreads, 0, s>>>(p->sell_ptr, p->sell_c16, p->n_slices,
                                                                        p->sell_cuptr, p->sell_cu);
  FEMK_CUDA_TRY(cudaGetLastError());
  FEMK_CUDA_TRY(cudaStreamSynchronize(s));
  return FEMK_OK;
}

// Assembly stream of the parametric assembly (femk_assemble): the geometry of a mesh does not change
// between assemblies, only the coefficient does, so for every (row, incident element) pair the plan
// keeps the row of the element's unit-coefficient stiffness matrix and the positions of the
// element's columns in the CSR row, in a sliced layout: slice s holds rows 32s..32s+31, entry k of
// row 32s + l at astr_ptr[s] + 32 k + l (width = the slice's largest incidence count; Dirichlet rows
// count 0). Per entry: the element (-1 = padding), ND FP64 stiffness values in ND planes of
// astr_len entries, and ND column positions (one byte each, 0xff for a Dirichlet column) padded to
// a multiple of 4 bytes. The load of every free row (the integral of its basis function) is kept too.
__global__ void k_astream_width(const int32_t* __restrict__ inc_ptr, const uint8_t* __restrict__ dmask, int64_t n,
                                int64_t nslices, int64_t* __restrict__ len) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t sl = warp; sl < nslices; sl += nwarps) {
    const int64_t row = sl * 32 + lane;
    int w = (row < n && !dmask[row]) ? inc_ptr[row + 1] - inc_ptr[row] : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) w = max(w, __shfl_xor_sync(0xffffffffu, w, o));
    if (lane == 0) len[sl] = (int64_t)w * 32;
  }
}

template <int ND>
__global__ void k_astream_fill(const double* __restrict__ xyz, const int32_t* __restrict__ cells,
                               const int32_t* __restrict__ inc_ptr, const int32_t* __restrict__ inc_elem,
                               const int32_t* __restrict__ indptr, const int32_t* __restrict__ indices,
                               const uint8_t* __restrict__ dmask, int64_t n, int64_t nslices,
                               const int64_t* __restrict__ aptr, int64_t alen, int32_t* __restrict__ ae,
                               double* __restrict__ ak, uint8_t* __restrict__ apos, double* __restrict__ aload,
                               int* __restrict__ err) {
  constexpr int NV = Cell<ND>::NV, PB = (ND + 3) / 4 * 4;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nslices * 32;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t sl = t >> 5, row = t;
    const int lane = (int)(t & 31);
    const int64_t a0 = aptr[sl], w = (aptr[sl + 1] - a0) >> 5;
    const bool free_row = row < n && !dmask[row];
    const int32_t j0 = free_row ? inc_ptr[row] : 0;
    const int32_t cnt = free_row ? inc_ptr[row + 1] - j0 : 0;
    const int32_t lo = free_row ? indptr[row] : 0, len = free_row ? indptr[row + 1] - lo : 0;
    double load = 0.0;
    for (int64_t k = 0; k < w; ++k) {
      const int64_t at = a0 + 32 * k + lane;
      if (k >= cnt) {
        ae[at] = -1;
#pragma unroll
        for (int c = 0; c < ND; ++c) ak[c * alen + at] = 0.0;
#pragma unroll
        for (int c = 0; c < PB; ++c) apos[at * PB + c] = 0xff;
        continue;
      }
      const int32_t e = inc_elem[j0 + k];
      int32_t dof[ND];
#pragma unroll
      for (int q = 0; q < ND; ++q) dof[q] = cells[(int64_t)e * ND + q];
      int a = 0;
#pragma unroll
      for (int q = 1; q < ND; ++q)
        if (dof[q] == (int32_t)row) a = q;
      Geom<NV> T;
      cell_geometry(xyz, dof, T);
      double VG[NV][NV];
      gram(T, VG);
      ae[at] = e;
#pragma unroll
      for (int c = 0; c < ND; ++c) {
        ak[c * alen + at] = khat<ND>(VG, a, c);
        uint8_t pos = 0xff;
        if (!dmask[dof[c]]) {
          const int32_t q = find_col(indices, lo, lo + len, dof[c]) - lo;
          if (q < len && indices[lo + q] == dof[c] && q < 0xff)
            pos = (uint8_t)q;
          else
            atomicOr(err, 32);
        }
        apos[at * PB + c] = pos;
      }
#pragma unroll
      for (int c = ND; c < PB; ++c) apos[at * PB + c] = 0xff;
      load += fhat<ND>(T.vol, a);
    }
    if (row < n) aload[row] = load;
  }
}

template <int ND>
int build_assembly_stream(femk_plan* p, cudaStream_t s) {
  constexpr int PB = (ND + 3) / 4 * 4;
  const int64_t n = p->n, ns = (n + 31) / 32;
  FEMK_CHECK_ARG(p->max_row < 0xff, "femk_plan_create: a CSR row has 255 or more entries");
  Temp len;
  FEMK_CUDA_TRY(cudaMalloc(&len.p, sizeof(int64_t) * (ns + 1)));
  FEMK_TRY(dev_alloc(&p->astr_ptr, ns + 1, s));
  const int sgrid = blocks_for(ns * 32, kThreads, p->n_sm * 64);
  k_astream_width<<<::femk::counted_launch() + sgrid, kThreads, 0, s>>>(p->inc_ptr, p->dmask, n, ns,
                                                                        (int64_t*)len.p);
  FEMK_TRY(scan_exclusive_i64((const int64_t*)len.p, p->astr_ptr, ns, s));
  FEMK_CUDA_TRY(cudaMemcpyAsync(&p->astr_len, p->astr_ptr + ns, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  FEMK_CUDA_TRY(cudaStreamSynchronize(s));
  const int64_t m = p->astr_len > 0 ? p->astr_len : 1;
  FEMK_TRY(dev_alloc(&p->astr_elem, m, s));
  FEMK_TRY(dev_alloc(&p->astr_k, ND * m, s));
  FEMK_TRY(dev_alloc(&p->astr_pos, PB * m, s));
  FEMK_TRY(dev_alloc(&p->astr_load, n, s));
  int* d_err = nullptr;
  FEMK_CUDA_TRY(cudaMalloc(&d_err, sizeof(int)));
  Temp eg;
  eg.p = d_err;
  FEMK_CUDA_TRY(cudaMemsetAsync(d_err, 0, sizeof(int), s));
  k_astream_fill<ND><<<::femk::counted_launch() + sgrid, kThreads, 0, s>>>(
      p->xyz, p->cells, p->inc_ptr, p->inc_elem, p->indptr, p->indices, p->dmask, n, ns, p->astr_ptr, m,
      p->astr_elem, p->astr_k, p->astr_pos, p->astr_load, d_err);
  FEMK_CUDA_TRY(cudaGetLastError());
  int h = 0;
  FEMK_TRY(read_err(d_err, s, &h));
  if (h) {
    set_error("femk_plan_create: assembly stream: a column is missing from its CSR row (corrupt connectivity?)");
    return FEMK_EBOUNDS;
  }
  return FEMK_OK;
}

int build_dirichlet(femk_plan* p, const uint8_t* user_mask, const int32_t* vptr, const int32_t* vinc, cudaStream_t s) {
  const int64_t n = p->n;
  FEMK_TRY(dev_alloc(&p->dmask, n, s));
  if (user_mask) {
    FEMK_CUDA_TRY(cudaMemcpyAsync(p->dmask, user_mask, n, cudaMemcpyDeviceToDevice, s));
  } else {
    FEMK_CUDA_TRY(cudaMemsetAsync(p->dmask, 0, n, s));
    const int grid = blocks_for(p->ntet * p->nv, kThreads, 65535 * 4);
    FEMK_BY_ND(p->nd, k_boundary<ND><<<::femk::counted_launch() + grid, kThreads, 0, s>>>(p->cells, p->ntet, vptr,
                                                                                         vinc, p->dmask));
    FEMK_CUDA_TRY(cudaGetLastError());
  }
  Temp flag, pos;
  FEMK_CUDA_TRY(cudaMalloc(&flag.p, sizeof(int64_t) * (n + 1)));
  FEMK_CUDA_TRY(cudaMalloc(&pos.p, sizeof(int64_t) * (n + 1)));
  k_mask_to_i64<<<::femk::counted_launch() + blocks_for(n, kThreads, 65535 * 4), kThreads, 0, s>>>(p->dmask, n, (int64_t*)flag.p);
  FEMK_TRY(scan_exclusive_i64((const int64_t*)flag.p, (int64_t*)pos.p, n, s));
  int64_t nd = 0;
  FEMK_CUDA_TRY(cudaMemcpyAsync(&nd, (int64_t*)pos.p + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  FEMK_CUDA_TRY(cudaStreamSynchronize(s));
  p->n_dir = nd;
  FEMK_TRY(dev_alloc(&p->dlist, nd, s));
  k_compact<<<::femk::counted_launch() + blocks_for(n, kThreads, 65535 * 4), kThreads, 0, s>>>(p->dmask, (const int64_t*)pos.p, n, p->dlist);
  FEMK_CUDA_TRY(cudaGetLastError());
  FEMK_CUDA_TRY(cudaStreamSynchronize(s));
  return FEMK_OK;
}

template <int NV>
int create_impl(femk_plan* p, const double* coords, const int32_t* tets, const uint8_t* mask, cudaStream_t s) {
  constexpr int NE = n_edges<NV>(), ND2 = NV + NE;
  int* d_err = nullptr;
  FEMK_CUDA_TRY(cudaMalloc(&d_err, sizeof(int)));
  Temp err_guard;
  err_guard.p = d_err;
  FEMK_CUDA_TRY(cudaMemsetAsync(d_err, 0, sizeof(int), s));
  int h_err = 0;

  k_validate_cells<NV><<<::femk::counted_launch() + blocks_for(p->ntet, kThreads, 65535 * 4), kThreads, 0, s>>>(
      tets, p->ntet, p->nvert, d_err);
  FEMK_CUDA_TRY(cudaGetLastError());
  FEMK_TRY(read_err(d_err, s, &h_err));
  if (h_err) {
    set_error("femk_plan_create: an element references a vertex outside [0, nvert) or repeats a vertex");
    return FEMK_EINVAL;
  }
  FEMK_TRY(dev_alloc(&p->xyz, p->nvert * 3, s));
  // vertex incidence (P1 connectivity): used by P2 numbering and by the boundary test
  int32_t* vptr = nullptr;
  int32_t* vinc = nullptr;
  FEMK_TRY(build_incidence<NV>(tets, p->ntet, p->nvert, &vptr, &vinc, d_err, s));
  FEMK_TRY(read_err(d_err, s, &h_err));
  if (h_err) {
    cudaFree(vptr);
    cudaFree(vinc);
    set_error("femk_plan_create: an element references a vertex outside [0, nvert)");
    return FEMK_EINVAL;
  }
  const int cgrid = blocks_for(p->nvert * 3, kThreads, 65535 * 4);
  if (p->order == 1) {
    p->n = p->nvert;
    FEMK_TRY(dev_alloc(&p->cells, p->ntet * NV, s));
    FEMK_CUDA_TRY(cudaMemcpyAsync(p->cells, tets, sizeof(int32_t) * p->ntet * NV, cudaMemcpyDeviceToDevice, s));
    FEMK_TRY(dev_alloc(&p->points, p->n * 3, s));
    k_copy_xyz<<<::femk::counted_launch() + cgrid, kThreads, 0, s>>>(coords, p->nvert, p->dim, p->xyz, p->points);
    p->inc_ptr = vptr;
    p->inc_elem = vinc;
  } else {
    k_copy_xyz<<<::femk::counted_launch() + cgrid, kThreads, 0, s>>>(coords, p->nvert, p->dim, p->xyz, nullptr);
    const int64_t m = p->ntet * NE;
    Temp first, isf, rank;
    FEMK_CUDA_TRY(cudaMalloc(&first.p, sizeof(int32_t) * m));
    FEMK_CUDA_TRY(cudaMalloc(&isf.p, sizeof(int64_t) * (m + 1)));
    FEMK_CUDA_TRY(cudaMalloc(&rank.p, sizeof(int64_t) * (m + 1)));
    k_edge_first<NV><<<::femk::counted_launch() + blocks_for(m, kThreads, 65535 * 4), kThreads, 0, s>>>(
        tets, p->ntet, vptr, vinc, (int32_t*)first.p, (int64_t*)isf.p, d_err);
    FEMK_CUDA_TRY(cudaGetLastError());
    FEMK_TRY(scan_exclusive_i64((const int64_t*)isf.p, (int64_t*)rank.p, m, s));
    int64_t nedge = 0;
    FEMK_CUDA_TRY(cudaMemcpyAsync(&nedge, (int64_t*)rank.p + m, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    FEMK_CUDA_TRY(cudaStreamSynchronize(s));
    p->n = p->nvert + nedge;
    if (p->n >= INT32_MAX) {
      cudaFree(vptr);
      cudaFree(vinc);
      set_error("femk_plan_create: too many DOFs for int32 indices");
      return FEMK_EINVAL;
    }
    FEMK_TRY(dev_alloc(&p->cells, p->ntet * ND2, s));
    FEMK_TRY(dev_alloc(&p->points, p->n * 3, s));
    FEMK_CUDA_TRY(cudaMemcpyAsync(p->points, p->xyz, sizeof(double) * p->nvert * 3, cudaMemcpyDeviceToDevice, s));
    k_p2_cells<NV><<<::femk::counted_launch() + blocks_for(m, kThreads, 65535 * 4), kThreads, 0, s>>>(
        tets, p->ntet, p->nvert, (const int32_t*)first.p, (const int64_t*)rank.p, p->xyz, p->cells, p->points);
    FEMK_CUDA_TRY(cudaGetLastError());
    FEMK_TRY(build_incidence<ND2>(p->cells, p->ntet, p->n, &p->inc_ptr, &p->inc_elem, d_err, s));
  }
  FEMK_TRY(read_err(d_err, s, &h_err));
  if (h_err) {
    if (vptr != p->inc_ptr) {
      cudaFree(vptr);
      cudaFree(vinc);
    }
    set_error("femk_plan_create: inconsistent connectivity (edge lookup failed)");
    return FEMK_EINVAL;
  }
  p->vstride = (p->n + 63) & ~int64_t(63);
  int st = FEMK_OK;
  FEMK_BY_ND(p->nd, st = build_pattern<ND>(p, d_err, &h_err, s));
  if (st == FEMK_OK) st = build_dirichlet(p, mask, vptr, vinc, s);
  if (st == FEMK_OK) FEMK_BY_ND(p->nd, st = build_assembly_stream<ND>(p, s));
  if (vptr != p->inc_ptr) {
    cudaFree(vptr);
    cudaFree(vinc);
  }
  return st;
}

}  // namespace
}  // namespace femk

extern "C" int femk_plan_destroy(femk_plan* p) {
  if (!p) return FEMK_OK;
  if (p->prof) femk_set_profiling(p, 0);
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(p->device);
  void* ptrs[] = {p->xyz,      p->points,    p->cells,     p->indptr,    p->indices,   p->slot,
                  p->diag,     p->dmask,     p->dlist,     p->inc_ptr,   p->inc_elem,  p->cols16,
                  p->work,     p->partials,  p->state,     p->work32,    p->vals32,    p->work64b,
                  p->sell_ptr, p->sell_cols, p->sell_c16,  p->sell_vals, p->sell_vals32,
                  p->bar,      p->batch_ws,  p->bicg_ws,   p->bicg_state, p->sell_cuptr, p->sell_cu,
                  p->coef_tmp, p->theta_ws, p->cmp_ws, p->gm_ws, p->dev_err, p->astr_ptr, p->astr_elem,
                  p->astr_k, p->astr_pos, p->astr_load, p->kcoef, p->mcells, p->kuhn};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  if (p->state_host) cudaFreeHost(p->state_host);
  if (p->cg_exec) cudaGraphExecDestroy(p->cg_exec);
  for (cudaEvent_t e : p->cg_ev)
    if (e) cudaEventDestroy(e);
  if (p->cg_stream) cudaStreamDestroy(p->cg_stream);
  if (p->mx_exec) cudaGraphExecDestroy(p->mx_exec);
  for (cudaEvent_t e : p->mx_ev)
    if (e) cudaEventDestroy(e);
  if (p->mx_stream) cudaStreamDestroy(p->mx_stream);
  if (p->mx_host) cudaFreeHost(p->mx_host);
  if (p->batch_exec) cudaGraphExecDestroy(p->batch_exec);
  if (p->batch_ev) cudaEventDestroy(p->batch_ev);
  if (p->batch_stream) cudaStreamDestroy(p->batch_stream);
  if (p->bicg_exec) cudaGraphExecDestroy(p->bicg_exec);
  for (cudaEvent_t e : p->bicg_ev)
    if (e) cudaEventDestroy(e);
  if (p->bicg_stream) cudaStreamDestroy(p->bicg_stream);
  if (p->bicg_host) cudaFreeHost(p->bicg_host);
  cudaSetDevice(cur);
  delete p;
  return FEMK_OK;
}

extern "C" void femk_plan_options_default(femk_plan_options* o) {
  if (!o) return;
  *o = femk_plan_options{};
  o->size = (int32_t)sizeof(femk_plan_options);
  o->solver_layout = 1;
  o->column_tables = 1;
  o->cols16 = 1;
  o->graph_replay = 1;
  o->l2_hints = -1;
  o->ring64 = -1;
  o->ring32 = -1;
  o->csr_lanes = 0;
  o->csr_rows = 0;
  o->sell_batch = 16;
  o->vec_blocks = 0;
  o->split_updates = 1;
  o->test_skip_arrival = -1;
  o->mixed_delta2 = 0.0;
  o->barrier_limit_ms = 0.0;
}

namespace {

bool ring_ok(int v) { return v == -1 || v == 0 || v == 14 || v == 18 || v == 24 || v == 28 || v == 38; }

// validate the options and copy them into the plan (before the build: the layout ones act there)
int apply_options(femk_plan* p, const femk_plan_options& o) {
  FEMK_CHECK_ARG(o.size == (int32_t)sizeof(femk_plan_options),
                 "femk_plan_create_ex: options.size mismatch (fill them with femk_plan_options_default)");
  FEMK_CHECK_ARG((o.solver_layout | 1) == 1 && (o.column_tables | 1) == 1 && (o.cols16 | 1) == 1 &&
                     (o.graph_replay | 1) == 1 && (o.split_updates | 1) == 1,
                 "femk_plan_create_ex: solver_layout, column_tables, cols16, graph_replay and split_updates are 0 or 1");
  FEMK_CHECK_ARG(o.l2_hints >= -1 && o.l2_hints <= 4, "femk_plan_create_ex: l2_hints must be in [-1, 4]");
  FEMK_CHECK_ARG(ring_ok(o.ring64) && ring_ok(o.ring32),
                 "femk_plan_create_ex: ring64 / ring32 must be -1, 0, 14, 18, 24, 28 or 38");
  const bool csr_auto = o.csr_lanes == 0 && o.csr_rows == 0;
  FEMK_CHECK_ARG(csr_auto || femk::with_spmv_cfg(o.csr_lanes, o.csr_rows, [](auto, auto) {}),
                 "femk_plan_create_ex: unsupported (csr_lanes, csr_rows) pair");
  FEMK_CHECK_ARG(o.sell_batch == 8 || o.sell_batch == 16, "femk_plan_create_ex: sell_batch must be 8 or 16");
  FEMK_CHECK_ARG(o.vec_blocks >= 0 && o.vec_blocks <= 8, "femk_plan_create_ex: vec_blocks must be in [0, 8]");
  FEMK_CHECK_ARG(o.test_skip_arrival >= -1, "femk_plan_create_ex: test_skip_arrival must be >= -1");
  FEMK_CHECK_ARG(o.mixed_delta2 >= 0.0 && o.mixed_delta2 < 1.0, "femk_plan_create_ex: mixed_delta2 must be in [0, 1)");
  FEMK_CHECK_ARG(o.barrier_limit_ms >= 0.0 && o.barrier_limit_ms <= 60000.0,
                 "femk_plan_create_ex: barrier_limit_ms must be in [0, 60000]");
  p->use_sell = o.solver_layout;
  p->sell_uni = o.column_tables;
  p->sell64_c16 = o.cols16;
  p->cg_graph = o.graph_replay;
  // measured on B200 (FP64 PCG to 1e-8): P1 128^3 48.7 ms with hints (mode 1) vs 52.0 ms without;
  // P2 64^3 117 ms without vs 168 ms with, so P2 plans stream without them
  p->l2_mode = o.l2_hints >= 0 ? o.l2_hints : (p->order == 1 ? 1 : 0);
  // bulk-copy SpMV rings, measured on B200 at P1 128^3 (solves to 1e-8): FP64 1 stage x 4 warps
  // (35.5 ms; 1 x 8: 35.0, 2 x 4: 43.4, 2 x 8: 38.2, thread-per-row: 44.0), FP32 1 stage x 4 warps
  // (23.6 ms; 1 x 8: 23.6, 2 x 4: 24.4, 2 x 8: 24.7); rows of at most 8 entries (2-D P1) get 2 x 8
  // (set after the build)
  p->bulk_cfg = o.ring64 >= 0 ? o.ring64 : 14;
  p->bulk32_cfg = o.ring32 >= 0 ? o.ring32 : 14;
  p->spmv_L = csr_auto ? 0 : o.csr_lanes;
  p->spmv_U = csr_auto ? 0 : o.csr_rows;
  p->sell_batch = o.sell_batch;
  p->vec_blocks = o.vec_blocks;
  p->cg_split = o.split_updates;
  p->skip_arrival = o.test_skip_arrival;
  p->mixed_delta2 = o.mixed_delta2;
  int khz = 0;
  cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, p->device);
  if (khz <= 0) khz = 2000000;
  const double ms = o.barrier_limit_ms > 0.0 ? o.barrier_limit_ms : 2000.0;
  p->barrier_spin = (long long)(ms * (double)khz);  // cycles at the maximum SM clock
  return FEMK_OK;
}

}  // namespace

extern "C" int femk_plan_create_ex(const double* coords_dev, int dim, int64_t nvert, const int32_t* cells_dev,
                                   int64_t ncell, int order, const uint8_t* dirichlet_mask_dev,
                                   const femk_plan_options* opts, void* stream, femk_plan** out) {
  femk::clear_error();
  FEMK_CHECK_ARG(out != nullptr, "femk_plan_create: out is NULL");
  *out = nullptr;
  FEMK_CHECK_ARG(coords_dev && cells_dev, "femk_plan_create: coordinates/cells is NULL");
  FEMK_CHECK_ARG(dim == 2 || dim == 3, "femk_plan_create: dim must be 2 (triangles) or 3 (tetrahedra)");
  FEMK_CHECK_ARG(order == 1 || order == 2, "femk_plan_create: order must be 1 or 2");
  const int nv = dim + 1;
  const int nd = order == 1 ? nv : nv * (nv + 1) / 2;  // P2: vertices + edges
  FEMK_CHECK_ARG(nvert >= nv && ncell >= 1, "femk_plan_create: empty mesh");
  FEMK_CHECK_ARG(ncell * nd * nd < INT32_MAX, "femk_plan_create: mesh too large for int32 slot map");
  FEMK_CHECK_ARG(nvert < INT32_MAX, "femk_plan_create: too many vertices");
  femk_plan_options o;
  femk_plan_options_default(&o);
  if (opts) o = *opts;
  cudaStream_t s = (cudaStream_t)stream;
  femk_plan* p = new femk_plan();
  cudaGetDevice(&p->device);
  cudaDeviceGetAttribute(&p->n_sm, cudaDevAttrMultiProcessorCount, p->device);
  p->order = order;
  p->dim = dim;
  p->nv = nv;
  p->nd = nd;
  int st = apply_options(p, o);
  if (st != FEMK_OK) {
    delete p;
    return st;
  }
  cudaDeviceGetAttribute(&p->coop, cudaDevAttrCooperativeLaunch, p->device);
  if (cudaMalloc(&p->dev_err, sizeof(int)) != cudaSuccess || cudaMemset(p->dev_err, 0, sizeof(int)) != cudaSuccess) {
    femk_plan_destroy(p);
    femk::set_error("femk_plan_create: device allocation failed");
    return FEMK_ENOMEM;
  }
  p->nvert = nvert;
  p->ntet = ncell;
  st = dim == 2 ? femk::create_impl<3>(p, coords_dev, cells_dev, dirichlet_mask_dev, s)
                : femk::create_impl<4>(p, coords_dev, cells_dev, dirichlet_mask_dev, s);
  if (st != FEMK_OK) {
    femk_plan_destroy(p);
    return st;
  }
  // rows of at most 8 entries (2-D P1 triangles) run on the 8-wide ring, where 2 stages x 8 warps
  // measured best on B200: 2-D P1 1024^2 PCG 109.7 ms vs 115.1 ms with 1 x 4
  if (p->max_row <= 8 && o.ring64 < 0) p->bulk_cfg = 28;
  *out = p;
  return FEMK_OK;
}

extern "C" int femk_plan_create_simplex(const double* coords_dev, int dim, int64_t nvert, const int32_t* cells_dev,
                                        int64_t ncell, int order, const uint8_t* dirichlet_mask_dev, void* stream,
                                        femk_plan** out) {
  return femk_plan_create_ex(coords_dev, dim, nvert, cells_dev, ncell, order, dirichlet_mask_dev, nullptr, stream,
                             out);
}

extern "C" int femk_plan_create(const double* xyz_dev, int64_t nvert, const int32_t* tets_dev, int64_t ntet,
                                int order, const uint8_t* dirichlet_mask_dev, void* stream, femk_plan** out) {
  return femk_plan_create_simplex(xyz_dev, 3, nvert, tets_dev, ntet, order, dirichlet_mask_dev, stream, out);
}

extern "C" int femk_plan_get_info(const femk_plan* p, femk_plan_info* out) {
  FEMK_CHECK_ARG(p && out, "femk_plan_get_info: NULL argument");
  out->order = p->order;
  out->ndof_local = p->nd;
  out->ntet = p->ntet;
  out->nvert = p->nvert;
  out->n = p->n;
  out->nnz = p->nnz;
  out->n_dirichlet = p->n_dir;
  out->cols16 = p->cols16 ? 1 : 0;
  out->device = p->device;
  out->sell_nnz = p->sell_cols ? p->sell_nnz : 0;
  out->batch_graph = p->batch_graph_used;
  out->sell_col_units = p->sell_cu ? p->sell_cu_len : (p->sell_cols ? p->sell_nnz : 0);
  out->dim = p->dim;
  return FEMK_OK;
}

extern "C" int femk_plan_export(const femk_plan* p, int32_t* indptr, int32_t* indices, int32_t* slot, int32_t* cells,
                                double* points, uint8_t* dmask, int32_t* diag, void* stream) {
  femk::clear_error();
  FEMK_CHECK_ARG(p, "femk_plan_export: plan is NULL");
  cudaStream_t s = (cudaStream_t)stream;
  const cudaMemcpyKind k = cudaMemcpyDeviceToDevice;
  if (indptr) FEMK_CUDA_TRY(cudaMemcpyAsync(indptr, p->indptr, sizeof(int32_t) * (p->n + 1), k, s));
  if (indices) FEMK_CUDA_TRY(cudaMemcpyAsync(indices, p->indices, sizeof(int32_t) * p->nnz, k, s));
  if (slot) FEMK_CUDA_TRY(cudaMemcpyAsync(slot, p->slot, sizeof(int32_t) * p->ntet * p->nd * p->nd, k, s));
  if (cells) FEMK_CUDA_TRY(cudaMemcpyAsync(cells, p->cells, sizeof(int32_t) * p->ntet * p->nd, k, s));
  if (points) FEMK_CUDA_TRY(cudaMemcpyAsync(points, p->points, sizeof(double) * p->n * 3, k, s));
  if (dmask) FEMK_CUDA_TRY(cudaMemcpyAsync(dmask, p->dmask, p->n, k, s));
  if (diag) FEMK_CUDA_TRY(cudaMemcpyAsync(diag, p->diag, sizeof(int32_t) * p->n, k, s));
  return FEMK_OK;
}
