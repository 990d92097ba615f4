// Parametric assembly: element geometry -> local stiffness -> CSR values -> symmetric Dirichlet
// elimination -> RHS.
//
// Replaces FemLinearSystem.evaluate (jno/trace/__init__.py:3612-3615) -> _assemble_at
// (jno/utils/solver/fem_native.py:3311-3316): per-cell jacfwd (fem_native.py:2333-2334) +
// segment_sum through the compress plan (fem_native.py:2318-2329) + _apply_dirichlet_symmetric
// (jno/utils/solver/fem_1d.py:667-686) + the residual's -1*v load (fem_native.py:2137-2181).
//
// Dirichlet semantics of the parametric route: entries in a Dirichlet row or column are stored as
// explicit zeros (they are never added), the diagonal slot of a Dirichlet row holds exactly 1
// (masked 0 + the appended unit triplet), b[d] = g[d], and free rows receive b -= A e.
//
// femk_assemble gathers instead of scattering: each CSR row is owned by one thread, which walks the
// row's incident elements (ascending element ids) in the plan's assembly stream -- per (row,
// element) pair the row of the element's unit-coefficient stiffness matrix and the positions of its
// columns in the CSR row, precomputed when the plan is built, since the geometry does not change
// between assemblies -- and adds k_e times that row, in that fixed order, into the row's values
// staged in shared memory; a block's rows are consecutive, so their values form one contiguous span
// that the block zeroes, accumulates and writes back with coalesced stores. The stream is laid out in
// 32-row slices (entry k of a row beside entry k of its 31 neighbours), so a warp's loads are
// coalesced; the only gather is the coefficient of each element. No atomics: the values and the load
// are the same bits on every run (the segment_sum of the reference has no defined order either).
#include <cmath>

#include "femk_element.cuh"
#include "femk_internal.cuh"

namespace femk {
namespace {

constexpr int kThreads = 128;

// One thread per row (blockDim.x consecutive rows per block, a multiple of 32 so that a warp walks
// one slice of the assembly stream); VALS: the CSR values are assembled (else the load alone, for
// matrix-free use). Shared memory: span_cap doubles, span_cap = the plan's largest block span.
template <int ND, bool VALS>
__global__ void __launch_bounds__(kThreads) k_assemble_stream(
    const int64_t* __restrict__ aptr, const int32_t* __restrict__ ae, const double* __restrict__ ak,
    const uint8_t* __restrict__ apos, int64_t alen, const double* __restrict__ aload,
    const int32_t* __restrict__ cells, const int32_t* __restrict__ indptr, const uint8_t* __restrict__ dmask,
    const int32_t* __restrict__ diag, int64_t n, int64_t ntet, int64_t nnz, const double* __restrict__ param,
    int mode, double scale, double f, const double* __restrict__ g, double* __restrict__ vals,
    double* __restrict__ b, int* __restrict__ err) {
  constexpr int PB = (ND + 3) / 4 * 4;
  extern __shared__ __align__(16) double asm_sv[];
  const int64_t r0 = (int64_t)blockIdx.x * blockDim.x;
  const int64_t r1 = r0 + blockDim.x < n ? r0 + blockDim.x : n;
  const int32_t base = VALS ? __ldg(indptr + r0) : 0;
  const int32_t span = VALS ? __ldg(indptr + r1) - base : 0;
  if (VALS) {
    for (int32_t k = threadIdx.x; k < span; k += blockDim.x) asm_sv[k] = 0.0;
    __syncthreads();
  }
  const int64_t row = r0 + threadIdx.x;
  if (row < r1) {
    if (__ldg(dmask + row)) {
      if (VALS) {
        const int32_t d = __ldg(diag + row) - base;
        if (FEMK_IN_BOUNDS(d, span, err)) asm_sv[d] = 1.0;
      }
      b[row] = g ? __ldg(g + row) : 0.0;
    } else {
      const int32_t lo = VALS ? __ldg(indptr + row) - base : 0;
      double bi = f * __ldg(aload + row);
      const int64_t sl = row >> 5;
      const int64_t a0 = __ldg(aptr + sl) + (row & 31);
      const int64_t w = (VALS || g) ? (__ldg(aptr + sl + 1) - __ldg(aptr + sl)) >> 5 : 0;
      // B pairs per trip: their stream loads, then their coefficient gathers, are issued together, so
      // a row's dependent element -> coefficient round trips overlap (the contributions are still
      // added in k order). Measured on B200: P1 128^3 0.455 ms with 2 pairs vs 0.481 ms with 4; P2
      // 64^3 0.649 ms with 2 vs 0.677 ms with 1 (each with the exp pass).
      constexpr int B = 2;
      for (int64_t k0 = 0; k0 < w; k0 += B) {
        int32_t e[B];
        uint32_t pw[B][PB / 4];
        double kh[B][ND];
#pragma unroll
        for (int u = 0; u < B; ++u) {
          const int64_t at = a0 + 32 * (k0 + u);
          const bool live = k0 + u < w;
          e[u] = live ? __ldcs(ae + at) : -1;
#pragma unroll
          for (int q = 0; q < PB / 4; ++q)
            pw[u][q] = live ? __ldcs(reinterpret_cast<const uint32_t*>(apos + at * PB) + q) : 0u;
#pragma unroll
          for (int c = 0; c < ND; ++c) kh[u][c] = live ? __ldcs(ak + c * alen + at) : 0.0;
        }
        double kk[B];
#pragma unroll
        for (int u = 0; u < B; ++u) {
          if (e[u] >= 0 && !FEMK_IN_BOUNDS(e[u], ntet, err)) e[u] = -1;
          kk[u] = e[u] >= 0 ? coef_of(param, mode, scale, e[u]) : 0.0;  // e < 0: padding past the row's elements
        }
#pragma unroll
        for (int u = 0; u < B; ++u) {
          if (e[u] < 0) continue;
#pragma unroll
          for (int c = 0; c < ND; ++c) {
            const uint32_t pc = (pw[u][c / 4] >> (8 * (c % 4))) & 0xffu;
            const double kac = kk[u] * kh[u][c];
            if (pc != 0xffu) {
              if (VALS && FEMK_IN_BOUNDS(lo + (int32_t)pc, span, err)) asm_sv[lo + pc] += kac;
            } else if (g) {
              bi -= kac * __ldg(g + __ldg(cells + (int64_t)e[u] * ND + c));
            }
          }
        }
      }
      b[row] = bi;
    }
  }
  if (VALS) {
    __syncthreads();
    for (int32_t k = threadIdx.x; k < span; k += blockDim.x)
      if (FEMK_IN_BOUNDS(base + k, nnz, err)) vals[base + k] = asm_sv[k];
  }
}

// k_e of a nodal P1 parameter (coef_nodal, unscaled) for every element: the kernels that take a
// coefficient then read it as a P0 linear parameter (FEMK_COEF_LINEAR with the caller's scale)
template <int NV>
__global__ void k_nodal_coef(const int32_t* __restrict__ cells, int64_t ntet, const double* __restrict__ param,
                             int mode, double* __restrict__ ke) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ntet; c += (int64_t)gridDim.x * blockDim.x) {
    int32_t v[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i) v[i] = __ldg(cells + c * NV + i);
    ke[c] = coef_nodal<NV>(param, mode, 1.0, v);
  }
}

template <int ND>
__global__ void k_element_matrices(const double* __restrict__ xyz, const int32_t* __restrict__ cells, int64_t ntet,
                                   double* __restrict__ khat_out, double* __restrict__ fhat_out) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ntet; c += (int64_t)gridDim.x * blockDim.x) {
    int32_t dof[Cell<ND>::NV];
#pragma unroll
    for (int a = 0; a < Cell<ND>::NV; ++a) dof[a] = cells[c * ND + a];
    Geom<Cell<ND>::NV> T;
    cell_geometry(xyz, dof, T);
    double VG[Cell<ND>::NV][Cell<ND>::NV];
    gram(T, VG);
    if (khat_out) {
#pragma unroll
      for (int a = 0; a < ND; ++a)
#pragma unroll
        for (int bb = 0; bb < ND; ++bb) khat_out[(c * ND + a) * ND + bb] = khat<ND>(VG, a, bb);
    }
    if (fhat_out) {
#pragma unroll
      for (int a = 0; a < ND; ++a) fhat_out[c * ND + a] = fhat<ND>(T.vol, a);
    }
  }
}

// Theta-step operators of the linear first-order block M u' + A u = c (the transient assembly of
// jno/utils/solver/fem_native.py:2846-3110, the step of jno/utils/solver/backend_blocks.py:332-345):
//   S = M' + theta dt A',  R = M' - (1 - theta) dt A',  q = dt c'
// per element into the canonical CSR. M' is the consistent mass with Dirichlet rows and columns
// zeroed. A' keeps the Dirichlet columns of the free rows when `rows` (row replacement, the
// parametric route: c' = the load on free rows) and drops them into the lift otherwise (symmetric
// elimination, the non-parametric route: c' = load - A e). Dirichlet rows are set afterwards
// (k_theta_dirichlet: A' row = identity, M' row = 0, c'[d] = g[d]).
template <int ND>
__global__ void __launch_bounds__(kThreads) k_assemble_theta(
    const double* __restrict__ xyz, const int32_t* __restrict__ cells, int64_t ntet, const int32_t* __restrict__ slot,
    const uint8_t* __restrict__ dmask, const double* __restrict__ param, int mode, double scale, double f,
    const double* __restrict__ g, double theta, double dt, int rows, double* __restrict__ S, double* __restrict__ R,
    double* __restrict__ q) {
  const double ws = theta * dt, wr = -(1.0 - theta) * dt;
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ntet; c += (int64_t)gridDim.x * blockDim.x) {
    int32_t dof[ND];
#pragma unroll
    for (int a = 0; a < ND; ++a) dof[a] = __ldg(cells + c * ND + a);
    Geom<Cell<ND>::NV> T;
    cell_geometry(xyz, dof, T);
    double VG[Cell<ND>::NV][Cell<ND>::NV];
    gram(T, VG);
    const double k = coef_of(param, mode, scale, c);
    bool dir[ND];
#pragma unroll
    for (int a = 0; a < ND; ++a) dir[a] = __ldg(dmask + dof[a]) != 0;
    const int32_t* srow = slot + c * ND * ND;
#pragma unroll
    for (int a = 0; a < ND; ++a) {
      if (dir[a]) continue;
      double rhs = f * fhat<ND>(T.vol, a);
#pragma unroll
      for (int bb = 0; bb < ND; ++bb) {
        const double kab = k * khat<ND>(VG, a, bb);
        const int32_t sl = __ldg(srow + a * ND + bb);
        if (dir[bb]) {
          if (rows) {
            atomicAdd(S + sl, ws * kab);
            atomicAdd(R + sl, wr * kab);
          } else if (g) {
            rhs -= kab * __ldg(g + dof[bb]);
          }
        } else {
          const double mab = T.vol * mhat<ND>(a, bb);
          atomicAdd(S + sl, mab + ws * kab);
          atomicAdd(R + sl, mab + wr * kab);
        }
      }
      atomicAdd(q + dof[a], dt * rhs);
    }
  }
}

__global__ void k_theta_dirichlet(const int32_t* __restrict__ dlist, int64_t nd, const int32_t* __restrict__ diag,
                                  const double* __restrict__ g, double theta, double dt, double* __restrict__ S,
                                  double* __restrict__ R, double* __restrict__ q) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nd; t += (int64_t)gridDim.x * blockDim.x) {
    const int32_t d = dlist[t];
    S[diag[d]] = theta * dt;
    R[diag[d]] = -(1.0 - theta) * dt;
    q[d] = g ? dt * g[d] : 0.0;
  }
}

// Consistent mass M[a][b] = integral(phi_a phi_b) into the canonical CSR; with `zero_dirichlet`
// the Dirichlet rows and columns are left at zero (the transient block's M).
template <int ND>
__global__ void __launch_bounds__(kThreads) k_mass(const double* __restrict__ xyz, const int32_t* __restrict__ cells,
                                                   int64_t ntet, const int32_t* __restrict__ slot,
                                                   const uint8_t* __restrict__ dmask, double* __restrict__ m) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ntet; c += (int64_t)gridDim.x * blockDim.x) {
    int32_t dof[ND];
#pragma unroll
    for (int a = 0; a < ND; ++a) dof[a] = __ldg(cells + c * ND + a);
    Geom<Cell<ND>::NV> T;
    cell_geometry(xyz, dof, T);
    bool dir[ND];
#pragma unroll
    for (int a = 0; a < ND; ++a) dir[a] = dmask ? __ldg(dmask + dof[a]) != 0 : false;
    const int32_t* srow = slot + c * ND * ND;
#pragma unroll
    for (int a = 0; a < ND; ++a) {
      if (dir[a]) continue;
#pragma unroll
      for (int bb = 0; bb < ND; ++bb)
        if (!dir[bb]) atomicAdd(m + __ldg(srow + a * ND + bb), T.vol * mhat<ND>(a, bb));
    }
  }
}

// Lumped mass: m_i = sum_e integral(phi_i) over every element (no Dirichlet masking).
template <int ND>
__global__ void k_lumped_mass(const double* __restrict__ xyz, const int32_t* __restrict__ cells, int64_t ntet,
                              double* __restrict__ m) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ntet; c += (int64_t)gridDim.x * blockDim.x) {
    int32_t dof[ND];
#pragma unroll
    for (int a = 0; a < ND; ++a) dof[a] = cells[c * ND + a];
    Geom<Cell<ND>::NV> T;
    cell_geometry(xyz, dof, T);
#pragma unroll
    for (int a = 0; a < ND; ++a) atomicAdd(m + dof[a], fhat<ND>(T.vol, a));
  }
}

// grad[c] = -k'_c (m o lam)_e^T K_hat_e (m o u)_e ; k'_c = dk/dparam_c
template <int ND>
__global__ void k_adjoint(const double* __restrict__ xyz, const int32_t* __restrict__ cells, int64_t ntet,
                          const uint8_t* __restrict__ dmask, const double* __restrict__ param, int mode, double scale,
                          const double* __restrict__ u, const double* __restrict__ lam, double* __restrict__ grad) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ntet; c += (int64_t)gridDim.x * blockDim.x) {
    int32_t dof[ND];
    double ue[ND], le[ND];
#pragma unroll
    for (int a = 0; a < ND; ++a) {
      dof[a] = __ldg(cells + c * ND + a);
      const bool d = __ldg(dmask + dof[a]) != 0;
      ue[a] = d ? 0.0 : __ldg(u + dof[a]);
      le[a] = d ? 0.0 : __ldg(lam + dof[a]);
    }
    Geom<Cell<ND>::NV> T;
    cell_geometry(xyz, dof, T);
    double VG[Cell<ND>::NV][Cell<ND>::NV];
    gram(T, VG);
    double acc = 0.0;
#pragma unroll
    for (int a = 0; a < ND; ++a) {
      double row = 0.0;
#pragma unroll
      for (int bb = 0; bb < ND; ++bb) row += khat<ND>(VG, a, bb) * ue[bb];
      acc += le[a] * row;
    }
    const double dk = mode == 0 ? scale * exp(__ldg(param + c)) : scale;
    grad[c] = -dk * acc;
  }
}

// Nodal P1 parameter: the element's dJ/dk_e = -(m o lam)^T K_hat (m o u) spread onto its NV
// vertex values by dk_e/dp_i (linear: scale / NV; exp with the degree-2 rule, L_q = a S + (b - a) p_q:
// scale / NV * (a sum_q exp(L_q) + (b - a) exp(L_i))). grad f64[nvert] must start at zero.
template <int NV>
__global__ void k_adjoint_nodal(const double* __restrict__ xyz, const int32_t* __restrict__ cells, int64_t ntet,
                                const uint8_t* __restrict__ dmask, const double* __restrict__ param, int mode,
                                double scale, const double* __restrict__ u, const double* __restrict__ lam,
                                double* __restrict__ grad) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ntet; c += (int64_t)gridDim.x * blockDim.x) {
    int32_t dof[NV];
    double ue[NV], le[NV], pv[NV];
#pragma unroll
    for (int a = 0; a < NV; ++a) {
      dof[a] = __ldg(cells + c * NV + a);
      const bool d = __ldg(dmask + dof[a]) != 0;
      ue[a] = d ? 0.0 : __ldg(u + dof[a]);
      le[a] = d ? 0.0 : __ldg(lam + dof[a]);
      pv[a] = __ldg(param + dof[a]);
    }
    Geom<NV> T;
    cell_geometry(xyz, dof, T);
    double VG[NV][NV];
    gram(T, VG);
    double acc = 0.0;
#pragma unroll
    for (int a = 0; a < NV; ++a) {
      double row = 0.0;
#pragma unroll
      for (int bb = 0; bb < NV; ++bb) row += khat<NV>(VG, a, bb) * ue[bb];
      acc += le[a] * row;
    }
    double dk[NV];
    if (mode == FEMK_COEF_NODAL_LINEAR) {
#pragma unroll
      for (int i = 0; i < NV; ++i) dk[i] = NodalRule<NV>::w * scale;
    } else {
      constexpr double qa = NodalRule<NV>::a, qb = NodalRule<NV>::b;
      double S = 0.0;
#pragma unroll
      for (int i = 0; i < NV; ++i) S += pv[i];
      double e[NV], es = 0.0;
#pragma unroll
      for (int i = 0; i < NV; ++i) {
        e[i] = exp(qa * S + (qb - qa) * pv[i]);
        es += e[i];
      }
#pragma unroll
      for (int i = 0; i < NV; ++i) dk[i] = NodalRule<NV>::w * scale * (qa * es + (qb - qa) * e[i]);
    }
#pragma unroll
    for (int i = 0; i < NV; ++i) atomicAdd(grad + dof[i], -acc * dk[i]);
  }
}

// Vector-Jacobian product of femk_assemble with respect to its parameter: given the cotangents
// gv of the values and gb of the load, S_e = sum_{a,b free} gv[slot(e,a,b)] K_hat_ab
// - sum_{a free, b Dirichlet} gb[a] K_hat_ab g[b] (the lift b -= A e g), and d(vals, b)/dparam_e
// = dk_e/dparam_e times that pattern. P0 modes: grad[e] = dk_e S_e (one write per element).
template <int ND>
__device__ __forceinline__ double vjp_sum(const double (&VG)[Cell<ND>::NV][Cell<ND>::NV], const int32_t (&dof)[ND],
                                          const bool (&dir)[ND], const int32_t* __restrict__ srow,
                                          const double* __restrict__ gv, const double* __restrict__ gb,
                                          const double* __restrict__ g) {
  double acc = 0.0;
#pragma unroll
  for (int a = 0; a < ND; ++a) {
    if (dir[a]) continue;
    const double gba = (gb && g) ? __ldg(gb + dof[a]) : 0.0;
#pragma unroll
    for (int bb = 0; bb < ND; ++bb) {
      const double kab = khat<ND>(VG, a, bb);
      if (!dir[bb]) {
        if (gv) acc += __ldg(gv + __ldg(srow + a * ND + bb)) * kab;
      } else if (gb && g) {
        acc -= gba * kab * __ldg(g + dof[bb]);
      }
    }
  }
  return acc;
}

template <int ND>
__global__ void __launch_bounds__(kThreads) k_assemble_vjp(const double* __restrict__ xyz,
                                                           const int32_t* __restrict__ cells, int64_t ntet,
                                                           const int32_t* __restrict__ slot,
                                                           const uint8_t* __restrict__ dmask,
                                                           const double* __restrict__ param, int mode, double scale,
                                                           const double* __restrict__ g, const double* __restrict__ gv,
                                                           const double* __restrict__ gb, double* __restrict__ grad) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ntet; c += (int64_t)gridDim.x * blockDim.x) {
    int32_t dof[ND];
    bool dir[ND];
#pragma unroll
    for (int a = 0; a < ND; ++a) {
      dof[a] = __ldg(cells + c * ND + a);
      dir[a] = __ldg(dmask + dof[a]) != 0;
    }
    Geom<Cell<ND>::NV> T;
    cell_geometry(xyz, dof, T);
    double VG[Cell<ND>::NV][Cell<ND>::NV];
    gram(T, VG);
    const double S = vjp_sum<ND>(VG, dof, dir, slot + c * ND * ND, gv, gb, g);
    const double dk = mode == FEMK_COEF_EXP ? scale * exp(__ldg(param + c)) : scale;
    grad[c] = dk * S;
  }
}

// Nodal P1 parameter: the element's S_e spread onto its NV vertex values by dk_e/dp_i (as in
// k_adjoint_nodal). grad f64[nvert] must start at zero.
template <int NV>
__global__ void __launch_bounds__(kThreads) k_assemble_vjp_nodal(
    const double* __restrict__ xyz, const int32_t* __restrict__ cells, int64_t ntet, const int32_t* __restrict__ slot,
    const uint8_t* __restrict__ dmask, const double* __restrict__ param, int mode, double scale,
    const double* __restrict__ g, const double* __restrict__ gv, const double* __restrict__ gb,
    double* __restrict__ grad) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ntet; c += (int64_t)gridDim.x * blockDim.x) {
    int32_t dof[NV];
    bool dir[NV];
    double pv[NV];
#pragma unroll
    for (int a = 0; a < NV; ++a) {
      dof[a] = __ldg(cells + c * NV + a);
      dir[a] = __ldg(dmask + dof[a]) != 0;
      pv[a] = __ldg(param + dof[a]);
    }
    Geom<NV> T;
    cell_geometry(xyz, dof, T);
    double VG[NV][NV];
    gram(T, VG);
    const double S = vjp_sum<NV>(VG, dof, dir, slot + c * NV * NV, gv, gb, g);
    double dk[NV];
    if (mode == FEMK_COEF_NODAL_LINEAR) {
#pragma unroll
      for (int i = 0; i < NV; ++i) dk[i] = NodalRule<NV>::w * scale;
    } else {
      constexpr double qa = NodalRule<NV>::a, qb = NodalRule<NV>::b;
      double Ssum = 0.0;
#pragma unroll
      for (int i = 0; i < NV; ++i) Ssum += pv[i];
      double e[NV], es = 0.0;
#pragma unroll
      for (int i = 0; i < NV; ++i) {
        e[i] = exp(qa * Ssum + (qb - qa) * pv[i]);
        es += e[i];
      }
#pragma unroll
      for (int i = 0; i < NV; ++i) dk[i] = NodalRule<NV>::w * scale * (qa * es + (qb - qa) * e[i]);
    }
#pragma unroll
    for (int i = 0; i < NV; ++i) atomicAdd(grad + dof[i], S * dk[i]);
  }
}

}  // namespace
}  // namespace femk

namespace femk {

// k_e = exp(param_e) once per element: the row-owner assembly and the matrix-free operator visit an
// element once per local DOF (and the operator once per CG step), each visit otherwise an FP64 exp
__global__ void k_exp_coef(const double* __restrict__ param, int64_t ntet, double* __restrict__ ke) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ntet; c += (int64_t)gridDim.x * blockDim.x)
    ke[c] = exp(param[c]);
}

int resolve_coef_exp(const femk_plan* pc, const double* param, int mode, cudaStream_t s, const double** param_out,
                     int* mode_out) {
  FEMK_TRY(resolve_coef(pc, param, mode, s, param_out, mode_out));
  if (*mode_out != FEMK_COEF_EXP) return FEMK_OK;
  femk_plan* p = const_cast<femk_plan*>(pc);
  if (!p->kcoef) FEMK_CUDA_TRY(cudaMalloc(&p->kcoef, sizeof(double) * (p->ntet > 0 ? p->ntet : 1)));
  k_exp_coef<<<counted_launch() + blocks_for(p->ntet, 256, p->n_sm * 16), 256, 0, s>>>(*param_out, p->ntet, p->kcoef);
  FEMK_CUDA_TRY(cudaGetLastError());
  *param_out = p->kcoef;
  *mode_out = FEMK_COEF_LINEAR;  // scale * kcoef[e] = scale * exp(param[e]), the same product
  return FEMK_OK;
}

int resolve_coef(const femk_plan* pc, const double* param, int mode, cudaStream_t s, const double** param_out,
                 int* mode_out) {
  *param_out = param;
  *mode_out = mode;
  if (mode != FEMK_COEF_NODAL_EXP && mode != FEMK_COEF_NODAL_LINEAR) return FEMK_OK;
  femk_plan* p = const_cast<femk_plan*>(pc);
  if (!p->coef_tmp) FEMK_CUDA_TRY(cudaMalloc(&p->coef_tmp, sizeof(double) * (p->ntet > 0 ? p->ntet : 1)));
  const int grid = blocks_for(p->ntet, 256, p->n_sm * 16);
  if (p->nd == 3)
    k_nodal_coef<3><<<counted_launch() + grid, 256, 0, s>>>(p->cells, p->ntet, param, mode, p->coef_tmp);
  else
    k_nodal_coef<4><<<counted_launch() + grid, 256, 0, s>>>(p->cells, p->ntet, param, mode, p->coef_tmp);
  FEMK_CUDA_TRY(cudaGetLastError());
  *param_out = p->coef_tmp;
  *mode_out = FEMK_COEF_LINEAR;
  return FEMK_OK;
}

}  // namespace femk

using namespace femk;

extern "C" int femk_assemble(const femk_plan* p, const double* param, int mode, double scale, double f,
                             const double* g, double* vals, double* b, void* stream) {
  clear_error();
  FEMK_CHECK_ARG(p && b, "femk_assemble: NULL plan/b");
  FEMK_CHECK_ARG(coef_mode_ok(p, mode, param),
                 "femk_assemble: unknown coef_mode, NULL param, or a nodal mode on a P2 plan");
  cudaStream_t s = (cudaStream_t)stream;
  if (vals || g)
    FEMK_TRY(resolve_coef_exp(p, param, mode, s, &param, &mode));
  else
    FEMK_TRY(resolve_coef(p, param, mode, s, &param, &mode));
  const int rows = p->asm_rows;
  const int grid = (int)((p->n + rows - 1) / rows);
  const size_t smem = vals ? (size_t)p->asm_span * sizeof(double) : 0;
  const int64_t alen = p->astr_len > 0 ? p->astr_len : 1;
  FEMK_BY_ND(p->nd, {
    if (vals) {
      auto kern = k_assemble_stream<ND, true>;
      FEMK_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      kern<<<::femk::counted_launch() + grid, rows, smem, s>>>(
          p->astr_ptr, p->astr_elem, p->astr_k, p->astr_pos, alen, p->astr_load, p->cells, p->indptr, p->dmask,
          p->diag, p->n, p->ntet, p->nnz, param, mode, scale, f, g, vals, b, p->dev_err);
    } else {
      k_assemble_stream<ND, false><<<::femk::counted_launch() + grid, rows, 0, s>>>(
          p->astr_ptr, p->astr_elem, p->astr_k, p->astr_pos, alen, p->astr_load, p->cells, p->indptr, p->dmask,
          p->diag, p->n, p->ntet, p->nnz, param, mode, scale, f, g, nullptr, b, p->dev_err);
    }
  });
  FEMK_CUDA_TRY(cudaGetLastError());
  return check_bounds(p, s, "femk_assemble");
}

extern "C" int femk_assemble_vjp(const femk_plan* p, const double* param, int mode, double scale, const double* g,
                                 const double* grad_vals, const double* grad_b, double* grad_param, void* stream) {
  clear_error();
  FEMK_CHECK_ARG(p && grad_param, "femk_assemble_vjp: NULL plan or grad_param");
  FEMK_CHECK_ARG(mode == FEMK_COEF_EXP || mode == FEMK_COEF_LINEAR || mode == FEMK_COEF_NODAL_EXP ||
                     mode == FEMK_COEF_NODAL_LINEAR,
                 "femk_assemble_vjp: coef_mode must be a P0 or nodal EXP/LINEAR mode (CONST has no parameter)");
  FEMK_CHECK_ARG(coef_mode_ok(p, mode, param), "femk_assemble_vjp: param is NULL or a nodal mode on a P2 plan");
  cudaStream_t s = (cudaStream_t)stream;
  const int grid = blocks_for(p->ntet, kThreads, p->n_sm * 16);
  if (mode == FEMK_COEF_NODAL_EXP || mode == FEMK_COEF_NODAL_LINEAR) {
    FEMK_CUDA_TRY(cudaMemsetAsync(grad_param, 0, sizeof(double) * p->nvert, s));
    if (p->nd == 3)
      k_assemble_vjp_nodal<3><<<::femk::counted_launch() + grid, kThreads, 0, s>>>(
          p->xyz, p->cells, p->ntet, p->slot, p->dmask, param, mode, scale, g, grad_vals, grad_b, grad_param);
    else
      k_assemble_vjp_nodal<4><<<::femk::counted_launch() + grid, kThreads, 0, s>>>(
          p->xyz, p->cells, p->ntet, p->slot, p->dmask, param, mode, scale, g, grad_vals, grad_b, grad_param);
  } else {
    FEMK_BY_ND(p->nd, k_assemble_vjp<ND><<<::femk::counted_launch() + grid, kThreads, 0, s>>>(
                          p->xyz, p->cells, p->ntet, p->slot, p->dmask, param, mode, scale, g, grad_vals, grad_b,
                          grad_param));
  }
  FEMK_CUDA_TRY(cudaGetLastError());
  return FEMK_OK;
}

extern "C" int femk_element_matrices(const femk_plan* p, double* khat_out, double* fhat_out, void* stream) {
  clear_error();
  FEMK_CHECK_ARG(p, "femk_element_matrices: NULL plan");
  cudaStream_t s = (cudaStream_t)stream;
  const int grid = blocks_for(p->ntet, kThreads, p->n_sm * 16);
  FEMK_BY_ND(p->nd, k_element_matrices<ND><<<::femk::counted_launch() + grid, kThreads, 0, s>>>(p->xyz, p->cells, p->ntet, khat_out, fhat_out));
  FEMK_CUDA_TRY(cudaGetLastError());
  return FEMK_OK;
}

extern "C" int femk_lumped_mass(const femk_plan* p, double* mass, void* stream) {
  clear_error();
  FEMK_CHECK_ARG(p && mass, "femk_lumped_mass: NULL argument");
  cudaStream_t s = (cudaStream_t)stream;
  FEMK_CUDA_TRY(cudaMemsetAsync(mass, 0, sizeof(double) * p->n, s));
  const int grid = blocks_for(p->ntet, kThreads, p->n_sm * 16);
  FEMK_BY_ND(p->nd, k_lumped_mass<ND><<<::femk::counted_launch() + grid, kThreads, 0, s>>>(p->xyz, p->cells, p->ntet, mass));
  FEMK_CUDA_TRY(cudaGetLastError());
  return FEMK_OK;
}

extern "C" int femk_adjoint_grad(const femk_plan* p, const double* param, int mode, double scale, const double* u,
                                 const double* lam, double* grad, void* stream) {
  clear_error();
  FEMK_CHECK_ARG(p && u && lam && grad, "femk_adjoint_grad: NULL argument");
  FEMK_CHECK_ARG(mode == FEMK_COEF_EXP || mode == FEMK_COEF_LINEAR || mode == FEMK_COEF_NODAL_EXP ||
                     mode == FEMK_COEF_NODAL_LINEAR,
                 "femk_adjoint_grad: coef_mode must be a P0 or nodal EXP/LINEAR mode");
  FEMK_CHECK_ARG(coef_mode_ok(p, mode, param) && (mode == FEMK_COEF_LINEAR || param),
                 "femk_adjoint_grad: param is NULL or a nodal mode on a P2 plan");
  cudaStream_t s = (cudaStream_t)stream;
  const int grid = blocks_for(p->ntet, kThreads, p->n_sm * 16);
  if (mode == FEMK_COEF_NODAL_EXP || mode == FEMK_COEF_NODAL_LINEAR) {
    FEMK_CUDA_TRY(cudaMemsetAsync(grad, 0, sizeof(double) * p->nvert, s));
    if (p->nd == 3)
      k_adjoint_nodal<3><<<::femk::counted_launch() + grid, kThreads, 0, s>>>(p->xyz, p->cells, p->ntet, p->dmask,
                                                                              param, mode, scale, u, lam, grad);
    else
      k_adjoint_nodal<4><<<::femk::counted_launch() + grid, kThreads, 0, s>>>(p->xyz, p->cells, p->ntet, p->dmask,
                                                                              param, mode, scale, u, lam, grad);
    FEMK_CUDA_TRY(cudaGetLastError());
    return FEMK_OK;
  }
  FEMK_BY_ND(p->nd, k_adjoint<ND><<<::femk::counted_launch() + grid, kThreads, 0, s>>>(p->xyz, p->cells, p->ntet, p->dmask, param, mode, scale, u, lam, grad));
  FEMK_CUDA_TRY(cudaGetLastError());
  return FEMK_OK;
}

extern "C" int femk_assemble_theta(const femk_plan* p, const double* param, int mode, double scale, double f,
                                   const double* g, double theta, double dt, int dirichlet, double* step_vals,
                                   double* rhs_vals, double* q, void* stream) {
  clear_error();
  FEMK_CHECK_ARG(p && step_vals && rhs_vals && q, "femk_assemble_theta: plan, step_vals, rhs_vals and q are required");
  FEMK_CHECK_ARG(coef_mode_ok(p, mode, param),
                 "femk_assemble_theta: unknown coef_mode, NULL param, or a nodal mode on a P2 plan");
  FEMK_CHECK_ARG(theta > 0.0 && theta <= 1.0, "femk_assemble_theta: theta must be in (0, 1]");
  FEMK_CHECK_ARG(dt > 0.0 && std::isfinite(dt), "femk_assemble_theta: dt must be positive and finite");
  FEMK_CHECK_ARG(dirichlet == FEMK_DIRICHLET_SYMMETRIC || dirichlet == FEMK_DIRICHLET_ROWS,
                 "femk_assemble_theta: dirichlet must be FEMK_DIRICHLET_SYMMETRIC or FEMK_DIRICHLET_ROWS");
  cudaStream_t s = (cudaStream_t)stream;
  FEMK_TRY(resolve_coef(p, param, mode, s, &param, &mode));
  FEMK_CUDA_TRY(cudaMemsetAsync(step_vals, 0, sizeof(double) * p->nnz, s));
  FEMK_CUDA_TRY(cudaMemsetAsync(rhs_vals, 0, sizeof(double) * p->nnz, s));
  FEMK_CUDA_TRY(cudaMemsetAsync(q, 0, sizeof(double) * p->n, s));
  const int grid = blocks_for(p->ntet, kThreads, p->n_sm * 16);
  const int rows = dirichlet == FEMK_DIRICHLET_ROWS;
  FEMK_BY_ND(p->nd, k_assemble_theta<ND><<<::femk::counted_launch() + grid, kThreads, 0, s>>>(
                        p->xyz, p->cells, p->ntet, p->slot, p->dmask, param, mode, scale, f, g, theta, dt, rows,
                        step_vals, rhs_vals, q));
  FEMK_CUDA_TRY(cudaGetLastError());
  if (p->n_dir > 0) {
    k_theta_dirichlet<<<::femk::counted_launch() + blocks_for(p->n_dir, 256, 65535), 256, 0, s>>>(
        p->dlist, p->n_dir, p->diag, g, theta, dt, step_vals, rhs_vals, q);
    FEMK_CUDA_TRY(cudaGetLastError());
  }
  return FEMK_OK;
}

extern "C" int femk_mass_matrix(const femk_plan* p, int zero_dirichlet, double* vals, void* stream) {
  clear_error();
  FEMK_CHECK_ARG(p && vals, "femk_mass_matrix: NULL argument");
  cudaStream_t s = (cudaStream_t)stream;
  FEMK_CUDA_TRY(cudaMemsetAsync(vals, 0, sizeof(double) * p->nnz, s));
  const int grid = blocks_for(p->ntet, kThreads, p->n_sm * 16);
  const uint8_t* dm = zero_dirichlet ? p->dmask : nullptr;
  FEMK_BY_ND(p->nd, k_mass<ND><<<::femk::counted_launch() + grid, kThreads, 0, s>>>(p->xyz, p->cells, p->ntet, p->slot,
                                                                                    dm, vals));
  FEMK_CUDA_TRY(cudaGetLastError());
  return FEMK_OK;
}
