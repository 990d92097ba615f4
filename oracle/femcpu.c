/*
 * femcpu.c -- CPU restatement (C, OpenMP, FP64) of the P1/P2 tetrahedral assembly -> Jacobi-PCG
 * path: the CPU baseline of the benchmark, the reference values of its full-size parity checks, and
 * a second CPU check of the numpy oracle. Test and benchmark infrastructure only: the product never
 * links it.
 *
 * It follows the same reference steps as the numpy oracle in this directory:
 *  - pattern: the compress-plan unique (row, col) set of all element DOF pairs, rows ascending,
 *    columns ascending within a row (jno/utils/solver/fem_utils.py:4049-4057);
 *  - values: k_e * integral(grad phi_a . grad phi_b) summed per (row, col) (segment_sum,
 *    jno/utils/solver/fem_native.py:2318-2329), closed forms from the Gram matrix V g_i . g_j of the
 *    barycentric gradients g of the affine map (fem_native.py:1480-1497);
 *  - load: b_a = f integral(phi_a) (the -1*v residual, fem_native.py:2137-2181);
 *  - symmetric Dirichlet elimination with u = 0: Dirichlet rows and columns stored as zeros, unit
 *    diagonal, b[d] = 0 (jno/utils/solver/fem_1d.py:667-686);
 *  - Jacobi inverse 1 / where(|d| > 1e-30, d, 1) (jno/precond.py:106-111);
 *  - preconditioned CG with jax.scipy.sparse.linalg.cg semantics (jax 0.10.1): stop when
 *    <r, r> <= max(tol^2 <b, b>, atol^2) or at maxiter (jno/solve.py:191-206).
 *
 * Parallel layout: every row is owned by one thread. Assembly gathers each row's contributions from
 * its incident elements (the vertex -> element incidence), so no two threads write one value and no
 * atomics are needed; the PCG loops are row-parallel with OpenMP reductions.
 *
 * Build: gcc -O3 -fopenmp -fPIC -shared femcpu.c -o _ref/... (oracle/build_cpu.py).
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

int femcpu_threads(void) { return omp_get_max_threads(); }

void femcpu_set_threads(int n) {
  if (n > 0) omp_set_num_threads(n);
}

/* DOF -> element incidence of cells i32[T, nd] (elements ascending per DOF): ptr i32[n+1], inc i32[nd T] */
int femcpu_incidence(int64_t n, int64_t T, int nd, const int32_t* cells, int32_t* ptr, int32_t* inc) {
  int64_t* cnt = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
  if (!cnt) return 1;
  for (int64_t t = 0; t < nd * T; ++t) cnt[cells[t] + 1] += 1;
  for (int64_t v = 0; v < n; ++v) cnt[v + 1] += cnt[v];
  for (int64_t v = 0; v <= n; ++v) ptr[v] = (int32_t)cnt[v];
  for (int64_t t = 0; t < nd * T; ++t) inc[cnt[cells[t]]++] = (int32_t)(t / nd);  /* element order kept */
  free(cnt);
  return 0;
}

/* the row's distinct columns (ascending) into cols; returns their count */
static int row_columns(int64_t row, int nd, const int32_t* cells, const int32_t* ptr, const int32_t* inc,
                       int32_t* cols, int cap) {
  int m = 0;
  for (int32_t j = ptr[row]; j < ptr[row + 1]; ++j) {
    const int32_t* t = cells + nd * (int64_t)inc[j];
    for (int a = 0; a < nd; ++a) {
      const int32_t c = t[a];
      int k = m - 1;
      while (k >= 0 && cols[k] > c) --k;
      if (k >= 0 && cols[k] == c) continue;
      if (m == cap) return -1;
      memmove(cols + k + 2, cols + k + 1, sizeof(int32_t) * (size_t)(m - k - 1));
      cols[k + 1] = c;
      ++m;
    }
  }
  return m;
}

/* CSR pattern: first call with indices == NULL fills indptr (i64 work in lens) and returns nnz */
int64_t femcpu_pattern(int64_t nv, int nd, const int32_t* cells, const int32_t* ptr, const int32_t* inc,
                       int32_t* indptr, int32_t* indices) {
  int64_t bad = 0;
  if (!indices) {
    int64_t* len = (int64_t*)malloc(sizeof(int64_t) * (size_t)nv);
    if (!len) return -1;
#pragma omp parallel for schedule(dynamic, 1024) reduction(+ : bad)
    for (int64_t i = 0; i < nv; ++i) {
      int32_t cols[512];
      const int m = row_columns(i, nd, cells, ptr, inc, cols, 512);
      if (m < 0) bad += 1;
      len[i] = m < 0 ? 0 : m;
    }
    int64_t s = 0;
    indptr[0] = 0;
    for (int64_t i = 0; i < nv; ++i) {
      s += len[i];
      indptr[i + 1] = (int32_t)s;
    }
    free(len);
    return bad ? -1 : s;
  }
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t i = 0; i < nv; ++i) row_columns(i, nd, cells, ptr, inc, indices + indptr[i], indptr[i + 1] - indptr[i]);
  return indptr[nv];
}

/* barycentric gradients g[4][3] and volume of the tet with vertex coordinates P[4][3] */
static inline double tet_grads(const double* x0, const double* x1, const double* x2, const double* x3,
                               double g[4][3]) {
  double e1[3], e2[3], e3[3];
  for (int k = 0; k < 3; ++k) {
    e1[k] = x1[k] - x0[k];
    e2[k] = x2[k] - x0[k];
    e3[k] = x3[k] - x0[k];
  }
  const double c23[3] = {e2[1] * e3[2] - e2[2] * e3[1], e2[2] * e3[0] - e2[0] * e3[2], e2[0] * e3[1] - e2[1] * e3[0]};
  const double c31[3] = {e3[1] * e1[2] - e3[2] * e1[1], e3[2] * e1[0] - e3[0] * e1[2], e3[0] * e1[1] - e3[1] * e1[0]};
  const double c12[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
  const double det = e1[0] * c23[0] + e1[1] * c23[1] + e1[2] * c23[2];
  const double inv = 1.0 / det;
  for (int k = 0; k < 3; ++k) {
    g[1][k] = c23[k] * inv;
    g[2][k] = c31[k] * inv;
    g[3][k] = c12[k] * inv;
    g[0][k] = -(g[1][k] + g[2][k] + g[3][k]);
  }
  return fabs(det) / 6.0;
}

/* basix P2 tetrahedron edges (jno/utils/solver/fem_topology.py:44): (2,3),(1,3),(1,2),(0,3),(0,2),(0,1) */
static const int kEdgeA[6] = {2, 1, 1, 0, 0, 0};
static const int kEdgeB[6] = {3, 3, 2, 3, 2, 1};

/* unit-coefficient stiffness K_hat[a][b] from the scaled Gram matrix VG[i][j] = V g_i . g_j:
 * P1 VG[a][b]; P2 (phi_i = l_i (2 l_i - 1), phi_e = 4 l_j l_k) the exact integrals of the products of
 * the basis gradients, int l_i l_j = V (1 + delta_ij) / 20 in 3-D */
static inline double khat(int nd, const double VG[4][4], int a, int b) {
  if (nd == 4) return VG[a][b];
  if (a < 4 && b < 4) return VG[a][b] * (a == b ? 0.6 : -0.2);
  if (a >= 4 && b >= 4) {
    const int i = kEdgeA[a - 4], j = kEdgeB[a - 4], l = kEdgeA[b - 4], m = kEdgeB[b - 4];
    return 0.8 * (VG[i][l] * (1 + (j == m)) + VG[i][m] * (1 + (j == l)) + VG[j][l] * (1 + (i == m)) +
                  VG[j][m] * (1 + (i == l)));
  }
  const int i = a < 4 ? a : b, e = a < 4 ? b - 4 : a - 4;
  const int j = kEdgeA[e], l = kEdgeB[e];
  return 4.0 * (VG[i][j] * (i == l ? 0.15 : -0.05) + VG[i][l] * (i == j ? 0.15 : -0.05));
}

/* unit-source load integral(phi_a): P1 V/4; P2 vertex -V/20, edge V/5 */
static inline double fhat(int nd, double vol, int a) {
  if (nd == 4) return 0.25 * vol;
  return a < 4 ? -0.05 * vol : 0.2 * vol;
}

/*
 * Parametric assembly of exp(logk_e) grad u . grad v - f v with u = 0 on the Dirichlet set, P1
 * (nd = 4) or P2 (nd = 10) tets: cells i32[T, nd] (the first 4 local DOFs are the vertices, whose
 * ids index xyz), vals f64[nnz] on the CSR pattern, b f64[n]. Row-gather: row i sums, in element
 * order, the contributions of its incident elements.
 */
void femcpu_assemble(int64_t n, int nd, const double* xyz, const int32_t* cells, const int32_t* ptr,
                     const int32_t* inc, const int32_t* indptr, const int32_t* indices, const uint8_t* dmask,
                     const double* logk, double f, double* vals, double* b) {
#pragma omp parallel for schedule(dynamic, 512)
  for (int64_t i = 0; i < n; ++i) {
    const int32_t lo = indptr[i], hi = indptr[i + 1];
    for (int32_t k = lo; k < hi; ++k) vals[k] = 0.0;
    if (dmask[i]) {
      for (int32_t k = lo; k < hi; ++k)
        if (indices[k] == i) vals[k] = 1.0;
      b[i] = 0.0;
      continue;
    }
    double bi = 0.0;
    for (int32_t j = ptr[i]; j < ptr[i + 1]; ++j) {
      const int64_t e = inc[j];
      const int32_t* t = cells + nd * e;
      double g[4][3], VG[4][4];
      const double vol = tet_grads(xyz + 3 * (int64_t)t[0], xyz + 3 * (int64_t)t[1], xyz + 3 * (int64_t)t[2],
                                   xyz + 3 * (int64_t)t[3], g);
      for (int p = 0; p < 4; ++p)
        for (int q = 0; q < 4; ++q) VG[p][q] = vol * (g[p][0] * g[q][0] + g[p][1] * g[q][1] + g[p][2] * g[q][2]);
      int a = 0;
      while (t[a] != i) ++a;
      const double k = exp(logk[e]);
      for (int c = 0; c < nd; ++c) {
        const int32_t col = t[c];
        if (dmask[col]) continue;
        int32_t s = lo;
        while (indices[s] != col) ++s;
        vals[s] += k * khat(nd, VG, a, c);
      }
      bi += f * fhat(nd, vol, a);
    }
    b[i] = bi;
  }
}

void femcpu_jacobi(int64_t n, const int32_t* indptr, const int32_t* indices, const double* vals, double* inv) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    double d = 0.0;
    for (int32_t k = indptr[i]; k < indptr[i + 1]; ++k)
      if (indices[k] == i) d += vals[k];
    inv[i] = 1.0 / (fabs(d) > 1e-30 ? d : 1.0);
  }
}

/*
 * Jacobi-PCG with jax cg semantics from x0 = x (overwritten with the solution). work f64[4n] (r, z,
 * p, q). Returns the iteration count; *relres = ||b - A x|| / (||b|| + 1e-30) of the result.
 */
int femcpu_pcg(int64_t n, const int32_t* indptr, const int32_t* indices, const double* vals, const double* b,
               const double* inv, double* x, double tol, double atol, int maxiter, double* work, double* relres) {
  double *r = work, *z = work + n, *p = work + 2 * n, *q = work + 3 * n;
  double gamma = 0.0, rr = 0.0, bb = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : gamma, rr, bb)
  for (int64_t i = 0; i < n; ++i) {
    double s = 0.0;
    for (int32_t k = indptr[i]; k < indptr[i + 1]; ++k) s += vals[k] * x[indices[k]];
    const double ri = b[i] - s, zi = inv[i] * ri;
    r[i] = ri;
    z[i] = zi;
    p[i] = zi;
    gamma += ri * zi;
    rr += ri * ri;
    bb += b[i] * b[i];
  }
  const double at2 = fmax(tol * tol * bb, atol * atol);
  int it = 0;
  while (rr > at2 && it < maxiter) {
    double pq = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : pq)
    for (int64_t i = 0; i < n; ++i) {
      double s = 0.0;
      for (int32_t k = indptr[i]; k < indptr[i + 1]; ++k) s += vals[k] * p[indices[k]];
      q[i] = s;
      pq += p[i] * s;
    }
    const double alpha = gamma / pq;
    double g2 = 0.0, r2 = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : g2, r2)
    for (int64_t i = 0; i < n; ++i) {
      x[i] += alpha * p[i];
      const double ri = r[i] - alpha * q[i], zi = inv[i] * ri;
      r[i] = ri;
      z[i] = zi;
      g2 += ri * zi;
      r2 += ri * ri;
    }
    const double beta = g2 / gamma;
    gamma = g2;
    rr = r2;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    ++it;
  }
  double w2 = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : w2)
  for (int64_t i = 0; i < n; ++i) {
    double s = 0.0;
    for (int32_t k = indptr[i]; k < indptr[i + 1]; ++k) s += vals[k] * x[indices[k]];
    w2 += (b[i] - s) * (b[i] - s);
  }
  if (relres) *relres = sqrt(w2) / (sqrt(bb) + 1e-30);
  return it;
}
