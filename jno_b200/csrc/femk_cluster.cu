// Matrix-free operator on element clusters staged in shared memory.
//
// y = A x with A the Dirichlet-eliminated stiffness, recomputed per element (the operator of
// k_matfree), but with the element loop cut into clusters of kCl consecutive elements, one block
// each. The plan records, once, every cluster's distinct DOFs (sorted) and each element's local
// slots in that list. A block stages the cluster's vertex coordinates, its x values (0 on Dirichlet
// DOFs) and the Dirichlet flags in shared memory, computes its elements' K_e x_e from there into
// per-(element, local dof) slots, then sums each cluster DOF's contributions in a fixed order
// (an inverse list built with the tables) and adds the sum to the global y once.
// On a structured Kuhn mesh 128 consecutive tetrahedra touch about 90 vertices against 512
// references, so global gathers and atomics drop about fivefold.
//
// Each element's row sums run in the order of k_matfree (b ascending), and y accumulates through
// atomics in both kernels, so the two agree to rounding.
//
// Opt-in (FEMK_MATFREE_CL=1): measured on B200 at P1 128^3, the matrix-free PCG step took 170.5 ms
// with the clusters against 139.8 ms with the per-element k_matfree, whose vertex reuse L1 already
// catches and whose global FP64 reductions do not wait; a first form with shared-memory FP64
// atomics for the cluster sums took 195.1 ms.
#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <thread>
#include <vector>

#include "femk_element.cuh"
#include "femk_internal.cuh"

namespace femk {
namespace {

constexpr int kCl = 128;          // elements per cluster = threads per block
constexpr int kClMaxSlots = 1024;  // distinct DOFs per cluster the shared-memory stage holds

template <int ND>
__global__ void __launch_bounds__(kCl) k_matfree_cl(const double* __restrict__ xyz, const int32_t* __restrict__ cl_ptr,
                                                    const int32_t* __restrict__ cl_dof,
                                                    const uint16_t* __restrict__ cl_loc,
                                                    const uint16_t* __restrict__ cl_off,
                                                    const uint16_t* __restrict__ cl_inv, int64_t ncl, int64_t ntet,
                                                    int64_t nvert, int cmax, const uint8_t* __restrict__ dmask,
                                                    const double* __restrict__ param, int mode, double scale,
                                                    const double* __restrict__ x, double* __restrict__ y,
                                                    const CgState* st) {
  constexpr int NV = Cell<ND>::NV;
  extern __shared__ __align__(16) double cl_smem[];
  if (st && st->done) return;
  double* xs = cl_smem;             // [3 cmax] coordinates of the vertex slots
  double* xv = xs + 3 * cmax;       // [cmax] x, 0 on Dirichlet DOFs
  double* ce = xv + cmax;           // [kCl ND] each element's contributions, (element, local dof)
  uint8_t* dm = reinterpret_cast<uint8_t*>(ce + kCl * ND);  // [cmax] Dirichlet flags
  for (int64_t c = blockIdx.x; c < ncl; c += gridDim.x) {
    const int32_t d0 = __ldg(cl_ptr + c), nc = __ldg(cl_ptr + c + 1) - d0;
    for (int j = threadIdx.x; j < nc; j += kCl) {
      const int32_t v = __ldg(cl_dof + d0 + j);
      const bool d = __ldg(dmask + v) != 0;
      dm[j] = d ? 1 : 0;
      xv[j] = d ? 0.0 : __ldg(x + v);
      if (v < nvert) {
#pragma unroll
        for (int k = 0; k < 3; ++k) xs[3 * j + k] = __ldg(xyz + (int64_t)v * 3 + k);
      }
    }
    __syncthreads();
    const int64_t e = c * kCl + threadIdx.x;
    if (e < ntet) {
      int loc[ND];
#pragma unroll
      for (int a = 0; a < ND; ++a) loc[a] = __ldg(cl_loc + e * ND + a);
      Geom<NV> T;
      cell_geometry_at(xs, loc, T);
      double VG[NV][NV];
      gram(T, VG);
      const double k = coef_of(param, mode, scale, e);
      double xe[ND];
#pragma unroll
      for (int a = 0; a < ND; ++a) xe[a] = xv[loc[a]];
#pragma unroll
      for (int a = 0; a < ND; ++a) {
        double s = 0.0;
#pragma unroll
        for (int b = 0; b < ND; ++b) s += khat<ND>(VG, a, b) * xe[b];
        ce[threadIdx.x * ND + a] = k * s;
      }
    }
    __syncthreads();
    // cluster DOF j: its contributions ce[cl_inv[o]] for o in [cl_off[j], cl_off[j + 1]), in a
    // fixed order (the cluster's (element, local dof) pairs sorted by slot)
    const uint16_t* off = cl_off + d0 + c;
    const uint16_t* inv = cl_inv + c * kCl * ND;
    for (int j = threadIdx.x; j < nc; j += kCl) {
      if (dm[j]) continue;
      double s = 0.0;
      for (int o = __ldg(off + j); o < __ldg(off + j + 1); ++o) s += ce[__ldg(inv + o)];
      atomicAdd(y + __ldg(cl_dof + d0 + j), s);
    }
    __syncthreads();  // the stage is refilled by the next cluster
  }
}

template <int ND>
int cluster_smem(int cmax) {
  return ((4 * cmax + kCl * ND) * (int)sizeof(double) + cmax + 15) / 16 * 16;
}

int cluster_smem_nd(int nd, int cmax) {
  int out = 0;
  FEMK_BY_ND(nd, out = cluster_smem<ND>(cmax));
  return out;
}

}  // namespace

// Build the cluster tables once per plan (host work on copies of the connectivity; called before
// any graph capture). Plans whose clusters exceed kClMaxSlots distinct DOFs keep k_matfree.
int ensure_clusters(femk_plan* p, cudaStream_t s) {
  if (p->cl_state != 0) return FEMK_OK;
  p->cl_state = -1;
  const char* on = std::getenv("FEMK_MATFREE_CL");
  if (!on || std::atoi(on) == 0) return FEMK_OK;
  const int nd = p->nd;
  const int64_t ntet = p->ntet, ncl = (ntet + kCl - 1) / kCl;
  std::vector<int32_t> cells((size_t)(ntet * nd));
  FEMK_CUDA_TRY(cudaMemcpyAsync(cells.data(), p->cells, sizeof(int32_t) * ntet * nd, cudaMemcpyDeviceToHost, s));
  FEMK_CUDA_TRY(cudaStreamSynchronize(s));
  std::vector<int32_t> cnt((size_t)ncl);
  std::vector<uint16_t> loc((size_t)(ntet * nd));
  std::vector<uint16_t> inv((size_t)(ncl * kCl * nd), 0);  // per cluster: (element, local dof) pairs by slot
  const int nth = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  std::vector<std::vector<uint16_t>> offs((size_t)nth);  // per cluster: nc + 1 slot offsets into its pairs
  std::vector<std::vector<int32_t>> lists((size_t)nth);
  std::vector<std::thread> pool;
  std::atomic<bool> too_wide{false};
  for (int t = 0; t < nth; ++t) {
    const int64_t c0 = ncl * t / nth, c1 = ncl * (t + 1) / nth;
    pool.emplace_back([&, t, c0, c1] {
      std::vector<int32_t> u;
      for (int64_t c = c0; c < c1; ++c) {
        const int64_t e0 = c * kCl, e1 = std::min<int64_t>(ntet, e0 + kCl);
        u.assign(cells.begin() + e0 * nd, cells.begin() + e1 * nd);
        std::sort(u.begin(), u.end());
        u.erase(std::unique(u.begin(), u.end()), u.end());
        if ((int64_t)u.size() > kClMaxSlots) too_wide = true;
        cnt[(size_t)c] = (int32_t)u.size();
        for (int64_t i = e0 * nd; i < e1 * nd; ++i)
          loc[(size_t)i] = (uint16_t)(std::lower_bound(u.begin(), u.end(), cells[(size_t)i]) - u.begin());
        lists[(size_t)t].insert(lists[(size_t)t].end(), u.begin(), u.end());
        if (too_wide) continue;
        // counting sort of the cluster's pairs by slot (pairs in (element, local dof) order)
        std::vector<uint16_t> o(u.size() + 1, 0);
        for (int64_t i = e0 * nd; i < e1 * nd; ++i) ++o[(size_t)loc[(size_t)i] + 1];
        for (size_t j = 0; j < u.size(); ++j) o[j + 1] = (uint16_t)(o[j + 1] + o[j]);
        std::vector<uint16_t> fill(o.begin(), o.end() - 1);
        uint16_t* ic = inv.data() + c * kCl * nd;
        for (int64_t i = e0 * nd; i < e1 * nd; ++i) ic[fill[(size_t)loc[(size_t)i]]++] = (uint16_t)(i - e0 * nd);
        offs[(size_t)t].insert(offs[(size_t)t].end(), o.begin(), o.end());
      }
    });
  }
  for (auto& th : pool) th.join();
  if (too_wide) return FEMK_OK;
  std::vector<int32_t> ptr((size_t)ncl + 1, 0);
  int cmax = 0;
  for (int64_t c = 0; c < ncl; ++c) {
    ptr[(size_t)c + 1] = ptr[(size_t)c] + cnt[(size_t)c];
    cmax = std::max(cmax, cnt[(size_t)c]);
  }
  std::vector<int32_t> dofs;
  dofs.reserve((size_t)ptr[(size_t)ncl]);
  for (auto& l : lists) dofs.insert(dofs.end(), l.begin(), l.end());
  std::vector<uint16_t> off;  // cluster c's nc + 1 offsets start at ptr[c] + c
  off.reserve((size_t)(ptr[(size_t)ncl] + ncl));
  for (auto& l : offs) off.insert(off.end(), l.begin(), l.end());
  FEMK_CUDA_TRY(cudaMalloc(&p->cl_ptr, sizeof(int32_t) * (ncl + 1)));
  FEMK_CUDA_TRY(cudaMalloc(&p->cl_dof, sizeof(int32_t) * std::max<size_t>(dofs.size(), 1)));
  FEMK_CUDA_TRY(cudaMalloc(&p->cl_loc, sizeof(uint16_t) * std::max<int64_t>(ntet * nd, 1)));
  FEMK_CUDA_TRY(cudaMalloc(&p->cl_off, sizeof(uint16_t) * off.size()));
  FEMK_CUDA_TRY(cudaMalloc(&p->cl_inv, sizeof(uint16_t) * inv.size()));
  FEMK_CUDA_TRY(cudaMemcpyAsync(p->cl_off, off.data(), sizeof(uint16_t) * off.size(), cudaMemcpyHostToDevice, s));
  FEMK_CUDA_TRY(cudaMemcpyAsync(p->cl_inv, inv.data(), sizeof(uint16_t) * inv.size(), cudaMemcpyHostToDevice, s));
  FEMK_CUDA_TRY(cudaMemcpyAsync(p->cl_ptr, ptr.data(), sizeof(int32_t) * (ncl + 1), cudaMemcpyHostToDevice, s));
  FEMK_CUDA_TRY(cudaMemcpyAsync(p->cl_dof, dofs.data(), sizeof(int32_t) * dofs.size(), cudaMemcpyHostToDevice, s));
  FEMK_CUDA_TRY(cudaMemcpyAsync(p->cl_loc, loc.data(), sizeof(uint16_t) * ntet * nd, cudaMemcpyHostToDevice, s));
  FEMK_CUDA_TRY(cudaStreamSynchronize(s));
  p->ncl = ncl;
  p->cl_max = cmax;
  // opt in to the stage size and read the occupancy now (never during a capture)
  const int smem = cluster_smem_nd(nd, cmax);
  int per_sm = 0;
  cudaError_t e = cudaSuccess;
  FEMK_BY_ND(nd, {
    auto kern = k_matfree_cl<ND>;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kCl, smem);
  });
  if (e != cudaSuccess || per_sm <= 0) {
    cudaGetLastError();
    return FEMK_OK;
  }
  p->cl_grid = (int)std::min<int64_t>(ncl, (int64_t)p->n_sm * std::min(per_sm, 16));
  p->cl_state = 1;
  return FEMK_OK;
}

// y += A x over the clusters (y zeroed by the caller); false when the plan has no cluster tables.
bool launch_matfree_cl(const femk_plan* p, const double* param, int mode, double scale, const double* x, double* y,
                       const CgState* st, cudaStream_t s) {
  if (p->cl_state != 1) return false;
  const int smem = cluster_smem_nd(p->nd, p->cl_max);
  FEMK_BY_ND(p->nd, k_matfree_cl<ND><<<counted_launch() + p->cl_grid, kCl, smem, s>>>(
                        p->xyz, p->cl_ptr, p->cl_dof, p->cl_loc, p->cl_off, p->cl_inv, p->ncl, p->ntet, p->nvert,
                        p->cl_max, p->dmask, param, mode, scale, x, y, st));
  return true;
}

}  // namespace femk
