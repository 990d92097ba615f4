// Per-element geometry and closed-form P1/P2 stiffness entries (device, FP64).
//
// Affine map of jno/utils/solver/fem_native.py:1480-1497: J = [x1-x0, ..., x_dim-x0] (columns),
// meas = |det J|, grad phi = dphi/dxi . J^-1. The rows of J^-1 are the barycentric gradients
// g1..g_dim (g0 = -(g1+...+g_dim)); they are formed from the adjugate (cross products of the edges
// of a tetrahedron, rotated edges of a triangle). Stiffness entries are the exact integrals of
// k grad phi_b . grad phi_a (the reference uses basix quadrature of degree 2 (P1) / 4 (P2), exact
// for these degree <= 2 integrands). Coordinates are stored x, y, z per vertex; a triangle reads
// x and y.
//
// An element is named by its local dof count ND: 3 / 6 = P1 / P2 triangle, 4 / 10 = P1 / P2
// tetrahedron (basix dof order: the vertices, then one midpoint per edge).
#pragma once

#include "../../include/femk.h"

#include <stdint.h>

namespace femk {

template <int ND>
struct Cell {
  static constexpr int NV = (ND == 3 || ND == 6) ? 3 : 4;  // vertices
  static constexpr int DIM = NV - 1;
  static constexpr bool P2 = ND == 6 || ND == 10;
};

// basix P2 tetrahedron edge order (jno/utils/solver/fem_topology.py:44):
// (2,3),(1,3),(1,2),(0,3),(0,2),(0,1)
__host__ __device__ constexpr int edge_a(int e) { return e == 0 ? 2 : (e <= 2 ? 1 : 0); }
__host__ __device__ constexpr int edge_b(int e) { return e == 0 || e == 1 || e == 3 ? 3 : (e == 2 || e == 4 ? 2 : 1); }
// basix P2 triangle edge order (jno/utils/solver/fem_topology.py:36): (1,2),(0,2),(0,1)
__host__ __device__ constexpr int tri_edge_a(int e) { return e == 0 ? 1 : 0; }
__host__ __device__ constexpr int tri_edge_b(int e) { return e == 2 ? 1 : 2; }
template <int NV>
__host__ __device__ constexpr int cell_edge_a(int e) {
  return NV == 3 ? tri_edge_a(e) : edge_a(e);
}
template <int NV>
__host__ __device__ constexpr int cell_edge_b(int e) {
  return NV == 3 ? tri_edge_b(e) : edge_b(e);
}

// local index of the edge between vertices j != m (compile-time when j and m are)
template <int NV>
__host__ __device__ constexpr int cell_edge_of(int j, int m) {
  for (int e = 0; e < (NV == 4 ? 6 : 3); ++e)
    if ((cell_edge_a<NV>(e) == j && cell_edge_b<NV>(e) == m) || (cell_edge_a<NV>(e) == m && cell_edge_b<NV>(e) == j))
      return e;
  return -1;
}

template <int NV>
struct Geom {
  double g[NV][NV - 1];  // barycentric gradients
  double vol;            // element measure: |det J| / 6 (tetrahedron), |det J| / 2 (triangle)
  double det;            // signed det J
};
using TetGeom = Geom<4>;

// Geometry from vertex coordinates P[i] (x, y, z of vertex i); the loaders below read them from
// the plan's coordinate array or from a shared-memory copy.
__device__ __forceinline__ void tet_geometry_of(const double (&P)[4][3], Geom<4>& G) {
  double e1[3], e2[3], e3[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    e1[k] = P[1][k] - P[0][k];
    e2[k] = P[2][k] - P[0][k];
    e3[k] = P[3][k] - P[0][k];
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

__device__ __forceinline__ void tri_geometry_of(const double (&P)[3][3], Geom<3>& G) {
  const double e1x = P[1][0] - P[0][0], e1y = P[1][1] - P[0][1];
  const double e2x = P[2][0] - P[0][0], e2y = P[2][1] - P[0][1];
  const double det = e1x * e2y - e1y * e2x;
  const double inv = 1.0 / det;
  G.g[1][0] = e2y * inv;
  G.g[1][1] = -e2x * inv;
  G.g[2][0] = -e1y * inv;
  G.g[2][1] = e1x * inv;
  G.g[0][0] = -(G.g[1][0] + G.g[2][0]);
  G.g[0][1] = -(G.g[1][1] + G.g[2][1]);
  G.det = det;
  G.vol = fabs(det) * 0.5;
}

__device__ __forceinline__ void tet_geometry(const double* __restrict__ xyz, int32_t v0, int32_t v1, int32_t v2,
                                             int32_t v3, TetGeom& G) {
  double P[4][3];
  const int32_t v[4] = {v0, v1, v2, v3};
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int k = 0; k < 3; ++k) P[i][k] = __ldg(xyz + (int64_t)v[i] * 3 + k);
  tet_geometry_of(P, G);
}

__device__ __forceinline__ void tri_geometry(const double* __restrict__ xyz, int32_t v0, int32_t v1, int32_t v2,
                                             Geom<3>& G) {
  double P[3][3];
  const int32_t v[3] = {v0, v1, v2};
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int k = 0; k < 2; ++k) P[i][k] = __ldg(xyz + (int64_t)v[i] * 3 + k);
  P[0][2] = P[1][2] = P[2][2] = 0.0;
  tri_geometry_of(P, G);
}

// the same from a coordinate array in shared memory (3 per local slot), vertices at slots loc[0..NV)
__device__ __forceinline__ void cell_geometry_at(const double* xs, const int* loc, Geom<4>& G) {
  double P[4][3];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int k = 0; k < 3; ++k) P[i][k] = xs[loc[i] * 3 + k];
  tet_geometry_of(P, G);
}
__device__ __forceinline__ void cell_geometry_at(const double* xs, const int* loc, Geom<3>& G) {
  double P[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int k = 0; k < 3; ++k) P[i][k] = k < 2 ? xs[loc[i] * 3 + k] : 0.0;
  tri_geometry_of(P, G);
}

// geometry of the element whose first NV local dofs (its vertices) are dof[0..NV)
__device__ __forceinline__ void cell_geometry(const double* __restrict__ xyz, const int32_t* dof, Geom<4>& G) {
  tet_geometry(xyz, dof[0], dof[1], dof[2], dof[3], G);
}
__device__ __forceinline__ void cell_geometry(const double* __restrict__ xyz, const int32_t* dof, Geom<3>& G) {
  tri_geometry(xyz, dof[0], dof[1], dof[2], G);
}

// Gram matrix of the barycentric gradients, scaled by the measure: VG[i][j] = V g_i . g_j
template <int NV>
__device__ __forceinline__ void gram(const Geom<NV>& T, double VG[NV][NV]) {
#pragma unroll
  for (int i = 0; i < NV; ++i)
#pragma unroll
    for (int j = i; j < NV; ++j) {
      double d = T.g[i][0] * T.g[j][0];
#pragma unroll
      for (int k = 1; k < NV - 1; ++k) d += T.g[i][k] * T.g[j][k];
      const double v = T.vol * d;
      VG[i][j] = v;
      VG[j][i] = v;
    }
}

// Unit-coefficient stiffness entry K_hat[a][b] from the scaled Gram matrix (a, b compile-time).
// P2 basis: phi_i = lambda_i (2 lambda_i - 1), phi_e = 4 lambda_j lambda_l on edge e = (j, l); with
// int lambda_i lambda_j = V (1 + delta_ij) / ((d+1)(d+2)) and int lambda_i = V / (d+1) in d dims.
template <int ND>
__device__ __forceinline__ double khat(const double VG[Cell<ND>::NV][Cell<ND>::NV], int a, int b) {
  constexpr int NV = Cell<ND>::NV;
  if (!Cell<ND>::P2) return VG[a][b];
  // tetrahedron / triangle moments of the P2 gradient products
  constexpr double vv_d = NV == 4 ? 0.6 : 1.0;          // int (4 l_i - 1)^2 / V
  constexpr double vv_o = NV == 4 ? -0.2 : -1.0 / 3.0;  // int (4 l_i - 1)(4 l_j - 1) / V
  constexpr double ee = NV == 4 ? 0.8 : 4.0 / 3.0;      // 16 int l_a l_b / V for a != b
  constexpr double ve_d = NV == 4 ? 0.15 : 1.0 / 3.0;   // int (4 l_i - 1) l_i / V
  constexpr double ve_o = NV == 4 ? -0.05 : 0.0;        // int (4 l_i - 1) l_l / V, l != i
  if (a < NV && b < NV) return VG[a][b] * (a == b ? vv_d : vv_o);
  if (a >= NV && b >= NV) {
    const int i = cell_edge_a<NV>(a - NV), j = cell_edge_b<NV>(a - NV);
    const int l = cell_edge_a<NV>(b - NV), m = cell_edge_b<NV>(b - NV);
    return ee * (VG[i][l] * (1 + (j == m)) + VG[i][m] * (1 + (j == l)) + VG[j][l] * (1 + (i == m)) +
                 VG[j][m] * (1 + (i == l)));
  }
  // vertex i against edge (j, l)
  const int i = a < NV ? a : b;
  const int e = a < NV ? b - NV : a - NV;
  const int j = cell_edge_a<NV>(e), l = cell_edge_b<NV>(e);
  const double cil = i == l ? ve_d : ve_o;
  const double cij = i == j ? ve_d : ve_o;
  return 4.0 * (VG[i][j] * cil + VG[i][l] * cij);
}

// P1 element product ye = K_hat xe (unit coefficient) straight from the vertex coordinates P, without
// the barycentric gradients or the Gram matrix. Tetrahedron: edges e_b = P_b - P_0, c_1 = e_2 x e_3,
// c_2 = e_3 x e_1, c_3 = e_1 x e_2 (det = e_1 . c_1, g_b = c_b / det) and w = sum_{b>=1} (x_b - x_0) c_b;
// then ye_a = V g_a . grad u = (c_a . w) / (6 |det|) for a >= 1, and ye_0 = -(ye_1 + ye_2 + ye_3)
// (the rows of K_hat sum to zero). Triangle: r_1 = (e_2y, -e_2x), r_2 = (-e_1y, e_1x),
// det = e_1x e_2y - e_1y e_2x, ye_a = (r_a . w) / (2 |det|). About 60 FP64 operations for a
// tetrahedron against ~140 through g and the Gram matrix; the same values up to rounding.
__device__ __forceinline__ void p1_apply(const double (&P)[4][3], const double (&xe)[4], double (&ye)[4]) {
  double e[3][3];
#pragma unroll
  for (int b = 0; b < 3; ++b)
#pragma unroll
    for (int k = 0; k < 3; ++k) e[b][k] = P[b + 1][k] - P[0][k];
  double c[3][3];
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    const double* u = e[(b + 1) % 3];
    const double* v = e[(b + 2) % 3];
    c[b][0] = u[1] * v[2] - u[2] * v[1];
    c[b][1] = u[2] * v[0] - u[0] * v[2];
    c[b][2] = u[0] * v[1] - u[1] * v[0];
  }
  const double det = e[0][0] * c[0][0] + e[0][1] * c[0][1] + e[0][2] * c[0][2];
  double w[3];
#pragma unroll
  for (int k = 0; k < 3; ++k)
    w[k] = (xe[1] - xe[0]) * c[0][k] + (xe[2] - xe[0]) * c[1][k] + (xe[3] - xe[0]) * c[2][k];
  const double s = 1.0 / (6.0 * fabs(det));
#pragma unroll
  for (int b = 0; b < 3; ++b) ye[b + 1] = (c[b][0] * w[0] + c[b][1] * w[1] + c[b][2] * w[2]) * s;
  ye[0] = -(ye[1] + ye[2] + ye[3]);
}
__device__ __forceinline__ void p1_apply(const double (&P)[3][3], const double (&xe)[3], double (&ye)[3]) {
  const double e1x = P[1][0] - P[0][0], e1y = P[1][1] - P[0][1];
  const double e2x = P[2][0] - P[0][0], e2y = P[2][1] - P[0][1];
  const double det = e1x * e2y - e1y * e2x;
  const double d1 = xe[1] - xe[0], d2 = xe[2] - xe[0];
  const double wx = d1 * e2y - d2 * e1y, wy = -d1 * e2x + d2 * e1x;  // w = d1 r_1 + d2 r_2
  const double s = 1.0 / (2.0 * fabs(det));
  ye[1] = (e2y * wx - e2x * wy) * s;
  ye[2] = (-e1y * wx + e1x * wy) * s;
  ye[0] = -(ye[1] + ye[2]);
}

// ye = K_hat xe for one element (unit coefficient) without forming the ND x ND matrix.
// P1: ye_a = sum_b VG[a][b] xe_b.
// P2: u = sum_a xe_a phi_a has grad u = sum_j G_j g_j with G_j = du/dlambda_j affine in the
// barycentric coordinates; using sum_l lambda_l = 1, G_j = sum_l H_jl lambda_l with H_jj = 3 x_j and
// H_jl = 4 x_(jl) - x_j (x_j the vertex values, x_(jl) the value at the midpoint of edge (j, l)).
// With int lambda_k lambda_l = V (1 + delta_kl) c, c = 1 / (NV (NV + 1)), and
// dphi_a/dlambda_j = sum_k A^a_jk lambda_k:
//   ye_a = c sum_jk A^a_jk Q_jk,  Q_jk = sum_m VG[j][m] (S_m + H_mk),  S_m = sum_l H_ml;
//   vertex i (A^i_jk = delta_ij (4 delta_ik - 1)):        ye_i    = c (4 Q_ii - sum_k Q_ik);
//   edge (i, m) (A_ik = 4 delta_mk, A_mk = 4 delta_ik):    ye_(im) = 4 c (Q_im + Q_mi).
// About NV^3 + 4 NV^2 FP64 operations against ~ND^2 (the matrix) plus forming K_hat; the same
// values as K_hat xe up to rounding.
template <int ND>
__device__ __forceinline__ void khat_apply(const double (&VG)[Cell<ND>::NV][Cell<ND>::NV], const double (&xe)[ND],
                                           double (&ye)[ND]) {
  constexpr int NV = Cell<ND>::NV;
  if constexpr (!Cell<ND>::P2) {
#pragma unroll
    for (int a = 0; a < ND; ++a) {
      double s = VG[a][0] * xe[0];
#pragma unroll
      for (int b = 1; b < ND; ++b) s = fma(VG[a][b], xe[b], s);
      ye[a] = s;
    }
  } else {
    constexpr double c = 1.0 / (NV * (NV + 1));
    auto H = [&](int m, int k) { return m == k ? 3.0 * xe[m] : 4.0 * xe[NV + cell_edge_of<NV>(m, k)] - xe[m]; };
    double S[NV];
#pragma unroll
    for (int m = 0; m < NV; ++m) {
      double t = 0.0;
#pragma unroll
      for (int l = 0; l < NV; ++l) t += H(m, l);
      S[m] = t;
    }
#pragma unroll
    for (int a = 0; a < ND; ++a) ye[a] = 0.0;
#pragma unroll
    for (int j = 0; j < NV; ++j) {
      double Q[NV], qs = 0.0;
#pragma unroll
      for (int k = 0; k < NV; ++k) {
        double q = 0.0;
#pragma unroll
        for (int m = 0; m < NV; ++m) q = fma(VG[j][m], S[m] + H(m, k), q);
        Q[k] = q;
        qs += q;
      }
      ye[j] = c * (4.0 * Q[j] - qs);
#pragma unroll
      for (int m = 0; m < NV; ++m)
        if (m != j) ye[NV + cell_edge_of<NV>(j, m)] += Q[m];
    }
#pragma unroll
    for (int e = 0; e < ND - NV; ++e) ye[NV + e] *= 4.0 * c;
  }
}

// Unit-source load integral(phi_a): P1 V / (d+1); P2 vertex V (2 - d) / ((d+1)(d+2)), edge
// 4 V / ((d+1)(d+2)) (a triangle's P2 vertex functions integrate to exactly 0)
template <int ND>
__device__ __forceinline__ double fhat(double vol, int a) {
  constexpr int NV = Cell<ND>::NV;
  if (ND == 4) return 0.25 * vol;
  if (ND == 3) return vol * (1.0 / 3.0);
  if (NV == 4) return a < 4 ? -0.05 * vol : 0.2 * vol;
  return a < 3 ? 0.0 : vol * (1.0 / 3.0);
}

// (1/V) integral over a d-simplex of prod_k lambda_k^{a_k} = d! prod_k a_k! / (sum_k a_k + d)!
__host__ __device__ constexpr double fact(int k) {
  double r = 1.0;
  for (int i = 2; i <= k; ++i) r *= i;
  return r;
}
__host__ __device__ constexpr double bary_moment(int d, int a0, int a1 = 0, int a2 = 0, int a3 = 0) {
  return fact(d) * fact(a0) * fact(a1) * fact(a2) * fact(a3) / fact(a0 + a1 + a2 + a3 + d);
}

// Unit-measure mass entry M_hat[a][b] = (1/V) integral(phi_a phi_b) (a, b compile-time), from the
// moments of the basis in barycentric coordinates: phi_i = lambda_i (2 lambda_i - 1), phi_e = 4
// lambda_j lambda_l on edge e = (j, l).
template <int ND>
__device__ __forceinline__ double mhat(int a, int b) {
  constexpr int NV = Cell<ND>::NV, D = Cell<ND>::DIM;
  if (!Cell<ND>::P2) return a == b ? bary_moment(D, 2) : bary_moment(D, 1, 1);
  if (a < NV && b < NV) {
    if (a == b) return 4.0 * bary_moment(D, 4) - 4.0 * bary_moment(D, 3) + bary_moment(D, 2);
    return 4.0 * bary_moment(D, 2, 2) - 4.0 * bary_moment(D, 2, 1) + bary_moment(D, 1, 1);
  }
  if (a >= NV && b >= NV) {
    const int i = cell_edge_a<NV>(a - NV), j = cell_edge_b<NV>(a - NV);
    const int l = cell_edge_a<NV>(b - NV), m = cell_edge_b<NV>(b - NV);
    const int shared = (i == l) + (i == m) + (j == l) + (j == m);
    if (shared == 2) return 16.0 * bary_moment(D, 2, 2);
    if (shared == 1) return 16.0 * bary_moment(D, 2, 1, 1);
    return 16.0 * bary_moment(D, 1, 1, 1, 1);
  }
  // vertex i against edge (j, l): 8 int lambda_i^2 lambda_j lambda_l - 4 int lambda_i lambda_j lambda_l
  const int i = a < NV ? a : b;
  const int e = a < NV ? b - NV : a - NV;
  const int j = cell_edge_a<NV>(e), l = cell_edge_b<NV>(e);
  if (i == j || i == l) return 8.0 * bary_moment(D, 3, 1) - 4.0 * bary_moment(D, 2, 1);
  return 8.0 * bary_moment(D, 2, 1, 1) - 4.0 * bary_moment(D, 1, 1, 1);
}

__device__ __forceinline__ double coef_of(const double* __restrict__ param, int mode, double scale, int64_t c) {
  if (mode == 2) return scale;
  const double p = __ldg(param + c);
  return mode == 0 ? scale * exp(p) : scale * p;
}

// Element coefficient of a nodal P1 parameter (one value per P1 vertex, interpolated linearly).
// P1 stiffness integrands are constant on an element, so K_e = V G * mean_q k(x_q):
//  * linear k (FEMK_COEF_NODAL_LINEAR): the quadrature mean of a linear field is the vertex mean;
//  * exp of a linear log-field (FEMK_COEF_NODAL_EXP): the symmetric degree-2 rule, the rule for
//    quadrature degree 2 that P1 forms are integrated with (jno/_fem.py:4551) -- on a tetrahedron
//    4 points with barycentric coordinates (b, a, a, a) and permutations, a = (5 - sqrt 5) / 20,
//    b = (5 + 3 sqrt 5) / 20; on a triangle 3 points (2/3, 1/6, 1/6) and permutations; equal weights.
//    Point q has L_q = a S + (b - a) p_q, S the vertex sum.
template <int NV>
struct NodalRule {
  static constexpr double a = NV == 4 ? 0.13819660112501051518 : 1.0 / 6.0;
  static constexpr double b = NV == 4 ? 0.58541019662496845446 : 2.0 / 3.0;
  static constexpr double w = 1.0 / NV;  // weight of a point in the mean
};

template <int NV>
__device__ __forceinline__ double coef_nodal(const double* __restrict__ param, int mode, double scale,
                                             const int32_t* v) {
  double p[NV], s = 0.0;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    p[i] = __ldg(param + v[i]);
    s += p[i];
  }
  if (mode == FEMK_COEF_NODAL_LINEAR) return scale * (NodalRule<NV>::w * s);
  constexpr double a = NodalRule<NV>::a, b = NodalRule<NV>::b;
  double e = 0.0;
#pragma unroll
  for (int i = 0; i < NV; ++i) e += exp(a * s + (b - a) * p[i]);
  return scale * (NodalRule<NV>::w * e);
}

}  // namespace femk
