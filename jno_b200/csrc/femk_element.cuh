// Per-element geometry and closed-form P1/P2 stiffness entries (device, FP64).
//
// Affine map of jno/utils/solver/fem_native.py:1480-1497: J = [x1-x0, x2-x0, x3-x0] (columns),
// meas = |det J|, grad phi = dphi/dxi . J^-1. The rows of J^-1 are the barycentric gradients
// g1..g3 (g0 = -(g1+g2+g3)); they are formed from the adjugate (cross products of the edges).
// Stiffness entries are the exact integrals of k grad phi_b . grad phi_a (the reference uses basix
// quadrature of degree 2 (P1) / 4 (P2), exact for these degree <= 2 integrands).
#pragma once

#include "../../include/femk.h"

#include <stdint.h>

namespace femk {

// basix P2 tetrahedron edge order (jno/utils/solver/fem_topology.py:44):
// (2,3),(1,3),(1,2),(0,3),(0,2),(0,1)
__host__ __device__ constexpr int edge_a(int e) { return e == 0 ? 2 : (e <= 2 ? 1 : 0); }
__host__ __device__ constexpr int edge_b(int e) { return e == 0 || e == 1 || e == 3 ? 3 : (e == 2 || e == 4 ? 2 : 1); }

struct TetGeom {
  double g[4][3];  // barycentric gradients
  double vol;      // |det J| / 6
  double det;      // signed det J
};

__device__ __forceinline__ void tet_geometry(const double* __restrict__ xyz, int32_t v0, int32_t v1, int32_t v2,
                                             int32_t v3, TetGeom& G) {
  double x0[3], e1[3], e2[3], e3[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    x0[k] = __ldg(xyz + (int64_t)v0 * 3 + k);
    e1[k] = __ldg(xyz + (int64_t)v1 * 3 + k) - x0[k];
    e2[k] = __ldg(xyz + (int64_t)v2 * 3 + k) - x0[k];
    e3[k] = __ldg(xyz + (int64_t)v3 * 3 + k) - x0[k];
  }
  const double c23[3] = {e2[1] * e3[2] - e2[2] * e3[1], e2[2] * e3[0] - e2[0] * e3[2], e2[0] * e3[1] - e2[1] * e3[0]};
  const double c31[3] = {e3[1] * e1[2] - e3[2] * e1[1], e3[2] * e1[0] - e3[0] * e1[2], e3[0] * e1[1] - e3[1] * e1[0]};
  const double c12[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
  const double det = e1[0] * c23[0] + e1[1] * c23[1] + e1[2] * c23[2];
  const double inv = 1.0 / det;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    G.g[1][k] = c23[k] * inv;
    G.g[2][k] = c31[k] * inv;
    G.g[3][k] = c12[k] * inv;
    G.g[0][k] = -(G.g[1][k] + G.g[2][k] + G.g[3][k]);
  }
  G.det = det;
  G.vol = fabs(det) * (1.0 / 6.0);
}

// Gram matrix of the barycentric gradients, scaled by the volume: VG[i][j] = V g_i . g_j
__device__ __forceinline__ void gram(const TetGeom& T, double VG[4][4]) {
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = i; j < 4; ++j) {
      const double v = T.vol * (T.g[i][0] * T.g[j][0] + T.g[i][1] * T.g[j][1] + T.g[i][2] * T.g[j][2]);
      VG[i][j] = v;
      VG[j][i] = v;
    }
}

// Unit-coefficient stiffness entry K_hat[a][b] from the scaled Gram matrix (a, b compile-time).
template <int ND>
__device__ __forceinline__ double khat(const double VG[4][4], int a, int b) {
  if (ND == 4) return VG[a][b];
  if (a < 4 && b < 4) return VG[a][b] * (a == b ? 0.6 : -0.2);
  if (a >= 4 && b >= 4) {
    const int i = edge_a(a - 4), j = edge_b(a - 4), l = edge_a(b - 4), m = edge_b(b - 4);
    return 0.8 * (VG[i][l] * (1 + (j == m)) + VG[i][m] * (1 + (j == l)) + VG[j][l] * (1 + (i == m)) +
                  VG[j][m] * (1 + (i == l)));
  }
  // vertex i against edge (j, l)
  const int i = a < 4 ? a : b;
  const int e = a < 4 ? b - 4 : a - 4;
  const int j = edge_a(e), l = edge_b(e);
  const double cil = i == l ? 0.15 : -0.05;
  const double cij = i == j ? 0.15 : -0.05;
  return 4.0 * (VG[i][j] * cil + VG[i][l] * cij);
}

// Unit-source load integral(phi_a)
template <int ND>
__device__ __forceinline__ double fhat(double vol, int a) {
  if (ND == 4) return 0.25 * vol;
  return a < 4 ? -0.05 * vol : 0.2 * vol;
}

__device__ __forceinline__ double coef_of(const double* __restrict__ param, int mode, double scale, int64_t c) {
  if (mode == 2) return scale;
  const double p = __ldg(param + c);
  return mode == 0 ? scale * exp(p) : scale * p;
}

// Element coefficient of a nodal P1 parameter (one value per P1 vertex, interpolated linearly).
// P1 stiffness integrands are constant on an element, so K_e = V G * mean_q k(x_q):
//  * linear k (FEMK_COEF_NODAL_LINEAR): the quadrature mean of a linear field is the vertex mean;
//  * exp of a linear log-field (FEMK_COEF_NODAL_EXP): the symmetric 4-point degree-2 tetrahedron
//    rule (points with barycentric coordinates (b, a, a, a) and its permutations,
//    a = (5 - sqrt 5) / 20, b = (5 + 3 sqrt 5) / 20, equal weights), the rule for quadrature degree 2
//    that P1 forms are integrated with (jno/_fem.py:4551).
__device__ __forceinline__ double coef_nodal(const double* __restrict__ param, int mode, double scale, int32_t v0,
                                             int32_t v1, int32_t v2, int32_t v3) {
  const double p0 = __ldg(param + v0), p1 = __ldg(param + v1), p2 = __ldg(param + v2), p3 = __ldg(param + v3);
  if (mode == FEMK_COEF_NODAL_LINEAR) return scale * (0.25 * (p0 + p1 + p2 + p3));
  constexpr double a = 0.13819660112501051518, b = 0.58541019662496845446;
  const double s = p0 + p1 + p2 + p3;
  const double e = exp(a * s + (b - a) * p0) + exp(a * s + (b - a) * p1) + exp(a * s + (b - a) * p2) +
                   exp(a * s + (b - a) * p3);
  return scale * (0.25 * e);
}

}  // namespace femk
