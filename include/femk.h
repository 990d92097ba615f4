/*
 * femk.h -- C ABI of the B200 (sm_100a) P1/P2 tetrahedral (and triangular) FEM assembly + Jacobi-PCG kernels.
 *
 * This is the drop-in boundary for jNO's hot path: parametric element assembly of
 * -div(k grad u) = f on Lagrange P1/P2 tetrahedra into the compress-plan CSR pattern, the Jacobi
 * preconditioner, and jax-cg-semantics preconditioned CG. Every entry point takes plain pointers
 * and sizes, returns an int status (FEMK_OK == 0) and never throws; the message of the last
 * failure on the calling thread is femk_last_error_string().
 *
 * Memory: arrays named *_dev are caller-owned DEVICE pointers on the plan's device; arrays named
 * *_host are host pointers. A plan owns its pattern arrays and its solver workspace and is
 * released with femk_plan_destroy. `stream` is a cudaStream_t passed as void* (NULL = default).
 * One plan may be used by one stream at a time.
 */
#ifndef FEMK_H
#define FEMK_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FEMK_OK 0
#define FEMK_EINVAL 1        /* bad argument (null pointer, size, out-of-range index) */
#define FEMK_ECUDA 2         /* a CUDA runtime call failed */
#define FEMK_ENOMEM 3        /* device allocation failed */
#define FEMK_NOT_CONVERGED 4 /* iteration cap reached above tolerance (solution still written) */
#define FEMK_NONFINITE 5     /* NaN/Inf met in a reduction */
#define FEMK_TIMEOUT 6       /* a bounded device-side wait gave up */
#define FEMK_EBOUNDS 7       /* an index check inside a kernel failed */
#define FEMK_BREAKDOWN 8     /* <p, A p> <= 0: operator not SPD */

/* coefficient modes for femk_assemble: k_e = coef_scale * g(param_e) */
#define FEMK_COEF_EXP 0      /* g = exp  : jno.np.exp(logk) * ...  (P0 log-conductivity) */
#define FEMK_COEF_LINEAR 1   /* g = id   : rho * ...               (P0 linear parameter) */
#define FEMK_COEF_CONST 2    /* g = 1    : param ignored (may be NULL) */
/* nodal P1 parameters (param f64[nvert], one value per P1 vertex; P1 plans only) */
#define FEMK_COEF_NODAL_EXP 3    /* k = exp(linear log-field), 4-point degree-2 quadrature mean */
#define FEMK_COEF_NODAL_LINEAR 4 /* k = linear field, element mean (exact) */

/* precision modes for femk_pcg_mixed */
#define FEMK_MIXED_RELIABLE 0 /* FP32 inner CG with FP64 reliable updates (no restart) */
#define FEMK_MIXED_RESTART 1  /* classic iterative refinement: restart FP32 CG per outer step */

/* Dirichlet treatment of the transient operator A' in femk_assemble_theta */
#define FEMK_DIRICHLET_SYMMETRIC 0 /* symmetric elimination + lift (the non-parametric transient route) */
#define FEMK_DIRICHLET_ROWS 1      /* row replacement, columns kept (the parametric transient route) */

typedef struct femk_plan femk_plan;

typedef struct femk_plan_info {
  int32_t order;      /* 1 or 2 */
  int32_t ndof_local; /* 4 or 10 (tetrahedra), 3 or 6 (triangles) */
  int64_t ntet;       /* elements (tetrahedra, or triangles on a 2-D plan) */
  int64_t nvert;      /* P1 vertices */
  int64_t n;          /* DOFs (rows) */
  int64_t nnz;        /* stored entries of the canonical CSR (= compress-plan nse) */
  int64_t n_dirichlet;
  int32_t cols16;     /* 1 when every column fits an int16 offset from its row (compact inner format) */
  int32_t device;
  int64_t sell_nnz;   /* stored entries of the solver's sliced-ELL copy (padding included), 0 if none */
  int32_t batch_graph; /* 1 when the last femk_pcg_batched ran as a replayed CUDA graph */
  int64_t sell_col_units; /* column entries the CG-step SpMV streams per product (int16 units when
                             cols16: per-slice tables, a shared-offset slice stored once) */
  int32_t dim;            /* 2 (triangles) or 3 (tetrahedra) */
} femk_plan_info;

/* Library version (major*10000 + minor*100 + patch). */
int femk_version(void);

/* 1 in the bounds-checked build (-DFEMK_BOUNDS_CHECK: kernels check their indexed accesses and the
 * entry points return FEMK_EBOUNDS when a check failed), 0 in the normal build. */
int femk_bounds_checked(void);

/* Number of CUDA kernels this library has launched in this process (all devices, all threads). */
int64_t femk_kernel_launches(void);

/* Message of the last failed call on this thread ("" if none). */
const char* femk_last_error_string(void);

/*
 * Build the assembly plan on the current device.
 *   xyz_dev   f64[nvert*3]  P1 vertex coordinates (x, y, z per vertex)
 *   tets_dev  i32[ntet*4]   P1 connectivity
 *   order     1 or 2        (P2 adds edge-midpoint DOFs numbered in first-encounter order)
 *   dirichlet_mask_dev  u8[n] or NULL: NULL = every node on a boundary facet (a facet owned by
 *             exactly one tet). For order 2 the DOF count n is only known after the build, so a
 *             P2 mask must come from a previous plan's export of the same mesh.
 * Replaces: jno/utils/solver/fem_native.py:218-288 (_get_mesh), fem_utils.py:1979-2044
 * (_promote_to_degree), fem_native.py:2264-2298 + fem_utils.py:4009-4057 (pattern hoist +
 * compress_plan), fem_native.py:2563-2636 (_boundary_node_ids) / jno/_fem.py:2695.
 */
int femk_plan_create(const double* xyz_dev, int64_t nvert, const int32_t* tets_dev, int64_t ntet,
                     int order, const uint8_t* dirichlet_mask_dev, void* stream, femk_plan** out);

/*
 * femk_plan_create for a simplex mesh of either dimension:
 *   dim 3: coords_dev f64[nvert*3], cells_dev i32[ncell*4] tetrahedra (= femk_plan_create);
 *   dim 2: coords_dev f64[nvert*2] (x, y per vertex), cells_dev i32[ncell*3] triangles. P2 adds
 *          one midpoint DOF per edge (basix triangle edge order (1,2),(0,2),(0,1),
 *          jno/utils/solver/fem_topology.py:36); boundary facets are the edges owned by one triangle.
 * The 2-D plan keeps 3 coordinates per node (z = 0): femk_plan_export writes points f64[n*3].
 * Every other entry point takes a 2-D plan as it is (ndof_local 3 / 6); the nodal modes work on
 * P1 triangles with the 3-point degree-2 rule. Replaces the dim == 2 branch of _get_mesh
 * (jno/utils/solver/fem_native.py:218-288, pts[:, :dim]) over Geometries.equi_distant_rect
 * (jno/domain/geometries.py:44-100) and the same pattern / facet steps as femk_plan_create.
 */
int femk_plan_create_simplex(const double* coords_dev, int dim, int64_t nvert, const int32_t* cells_dev,
                             int64_t ncell, int order, const uint8_t* dirichlet_mask_dev, void* stream,
                             femk_plan** out);

/*
 * Per-plan layout and tuning options of femk_plan_create_ex. femk_plan_options_default fills in the
 * defaults, which are what femk_plan_create / femk_plan_create_simplex use; the library reads no
 * environment variables. Layout options act when the plan is built; the others on every call that
 * uses the plan. Every field is validated at creation (FEMK_EINVAL for an unknown value). No
 * reference counterpart (jNO's assembly and solver have no such knobs).
 */
typedef struct femk_plan_options {
  int32_t size;           /* sizeof(femk_plan_options): set by femk_plan_options_default */
  int32_t solver_layout;  /* 1 (default): the CG loops multiply with a sliced-ELL (SELL-32) copy of the
                             operator; 0: with the canonical CSR itself (the plain method) */
  int32_t column_tables;  /* 1 (default): a slice whose 32 rows share one column-offset sequence stores it once */
  int32_t cols16;         /* 1 (default): int16 column offsets in the FP64 sliced-ELL stream when they fit */
  int32_t graph_replay;   /* 1 (default): CG / mixed chunks replayed as CUDA graphs; 0: launched one by one */
  int32_t l2_hints;       /* L2 eviction hints of the FP64 CG kernels: -1 (default) on for P1, off for P2;
                             0 off; 1 matrix evict-first, gathers and vectors evict-last; 2 matrix evict-first,
                             vectors evict-last; 3 vectors evict-last only; 4 as 1 with streaming matrix loads */
  int32_t ring64;         /* bulk-copy ring of the FP64 CG-step SpMV, 10 * stages + warps per block (14, 18,
                             24, 28, 38); -1 (default): 14, 28 for rows of at most 8 entries; 0: thread-per-row kernel */
  int32_t ring32;         /* the same for the FP32 step of femk_pcg_mixed; -1 (default): 14 */
  int32_t csr_lanes;      /* CSR SpMV lanes per row (4, 8, 16, 32); 0 (default): from the mean row length */
  int32_t csr_rows;       /* CSR rows in flight per lane group (1, 2, 4); 0 (default): with csr_lanes */
  int32_t sell_batch;     /* entries in flight per thread of the thread-per-row FP64 kernel: 8, or 16 (default;
                             32 on plans with int32 columns, such as 3-D P2) */
  int32_t vec_blocks;     /* blocks per SM of the FP64 CG vector kernels; 0 (default): one full wave */
  int32_t split_updates;  /* 1 (default): FP64 CG vector updates as r-update + direction/x-update kernels */
  int32_t test_skip_arrival; /* testing the bounded waits: the block with this index skips its first
                                grid-barrier arrival in femk_pcg_batched*, so every other block waits out
                                barrier_limit_ms and the call returns FEMK_TIMEOUT; -1 (default): none */
  double mixed_delta2;    /* reliable update of the mixed solvers once <r, r> fell by this factor; 0 (default): 1e-4 */
  double barrier_limit_ms; /* limit of each grid-barrier wait of femk_pcg_batched*, in milliseconds at the
                              maximum SM clock; 0 (default): 2000 */
} femk_plan_options;

void femk_plan_options_default(femk_plan_options* opts);

/* femk_plan_create_simplex with explicit options (NULL = the defaults). */
int femk_plan_create_ex(const double* coords_dev, int dim, int64_t nvert, const int32_t* cells_dev, int64_t ncell,
                        int order, const uint8_t* dirichlet_mask_dev, const femk_plan_options* opts, void* stream,
                        femk_plan** out);

int femk_plan_destroy(femk_plan* plan);

int femk_plan_get_info(const femk_plan* plan, femk_plan_info* out);

/*
 * Copy plan arrays into caller buffers (device pointers; each may be NULL to skip):
 *   indptr i32[n+1], indices i32[nnz]  canonical CSR (compress_plan(...)[0], fem_utils.py:4049-4053)
 *   slot   i32[ntet*nd*nd]             element -> CSR slot in (c, a, b) order (compress_plan inverse)
 *   cells  i32[ntet*nd]                global DOF per (cell, local dof) (fem_native.py:908-913)
 *   points f64[n*3]                    DOF coordinates (P2 midpoints = 0.5*xa + 0.5*xb)
 *   dirichlet_mask u8[n], diag_slot i32[n]
 */
int femk_plan_export(const femk_plan* plan, int32_t* indptr_dev, int32_t* indices_dev,
                     int32_t* slot_dev, int32_t* cells_dev, double* points_dev,
                     uint8_t* dirichlet_mask_dev, int32_t* diag_slot_dev, void* stream);

/*
 * Parametric assembly of  k_e * grad u . grad v - f v  with symmetric Dirichlet u = g.
 *   param_dev f64[ntet] (per-element P0 value) or f64[nvert] (nodal P1 modes), see FEMK_COEF_*;
 *   coef_scale multiplies k_e,
 *   f       constant source, g_dev f64[n] Dirichlet values or NULL (= 0),
 *   vals_dev f64[nnz] (canonical CSR values, explicit zeros kept) or NULL to assemble the load only
 *   (matrix-free use), b_dev f64[n].
 * Dirichlet rows/columns are zero, the diagonal 1, b[d] = g[d], and b -= A e carries g into the
 * free rows. Replaces: FemLinearSystem.evaluate (jno/trace/__init__.py:3612-3615) ->
 * _assemble_at (jno/utils/solver/fem_native.py:3311-3316): jacobian + residual + segment_sum +
 * _apply_dirichlet_symmetric (fem_1d.py:667-686).
 */
int femk_assemble(const femk_plan* plan, const double* param_dev, int coef_mode, double coef_scale,
                  double f, const double* g_dev, double* vals_dev, double* b_dev, void* stream);

/*
 * Vector-Jacobian product of femk_assemble with respect to its parameter (the reverse pass jax.grad
 * takes through the parametric assembly: segment_sum and the per-cell jacfwd, fem_native.py:2318-2334,
 * and the Dirichlet lift b -= A e g). Given cotangents grad_vals_dev f64[nnz] of the values and
 * grad_b_dev f64[n] of the load (either may be NULL = zero), grad_param_dev receives
 *   P0 modes: f64[ntet], grad[e] = dk_e/dparam_e * S_e,
 *   nodal modes: f64[nvert], grad[i] = sum over elements e holding vertex i of S_e * dk_e/dparam_i,
 *   S_e = sum_{a,b free} grad_vals[slot(e,a,b)] K_hat_e[a,b] - sum_{a free, b Dirichlet} grad_b[a] K_hat_e[a,b] g[b].
 * param, mode, scale and g are those of the femk_assemble call (CONST has no parameter: FEMK_EINVAL).
 */
int femk_assemble_vjp(const femk_plan* plan, const double* param_dev, int coef_mode, double coef_scale,
                      const double* g_dev, const double* grad_vals_dev, const double* grad_b_dev,
                      double* grad_param_dev, void* stream);

/*
 * Compact export of assembled values: the canonical CSR entries with |v| > 0, in CSR order (rows
 * ascending, columns ascending). Exact zeros (the zeroed Dirichlet rows and columns, values that
 * summed to 0) and NaNs are dropped.
 *   vals_dev f64[nnz] (from femk_assemble), indptr_out_dev i32[n+1],
 *   indices_out_dev i32[cap], vals_out_dev f64[cap], *nnz_out = kept entries.
 * The call waits on `stream` for the count (one 8-byte device-to-host read) and returns
 * FEMK_EINVAL without writing entries when it exceeds cap; cap = plan nnz always suffices.
 * Replaces compress_eager (jno/utils/solver/fem_utils.py:4063-4091) on the non-parametric linear
 * route (jno/utils/solver/fem_native.py:3371-3379).
 */
int femk_compact(const femk_plan* plan, const double* vals_dev, int32_t* indptr_out_dev, int32_t* indices_out_dev,
                 double* vals_out_dev, int64_t cap, int64_t* nnz_out, void* stream);

/* Unit-coefficient element matrices K_hat f64[ntet*nd*nd] and loads F_hat f64[ntet*nd]
 * (either may be NULL). Replaces the per-cell jacfwd of fem_native.py:2333-2334 for k = 1. */
int femk_element_matrices(const femk_plan* plan, double* khat_dev, double* fhat_dev, void* stream);

/* inv_diag[i] = 1 / where(|A_ii| > 1e-30, A_ii, 1).
 * Replaces matrix_diagonal (jno/utils/solver/linear.py:88-94) + _Jacobi.materialize (jno/precond.py:106-111). */
int femk_jacobi(const femk_plan* plan, const double* vals_dev, double* inv_diag_dev, void* stream);

/* Jacobi inverse diagonal of the matrix-free operator (same values as femk_jacobi on the
 * assembled matrix, summed per element instead of read from the CSR diagonal slot). */
int femk_jacobi_matfree(const femk_plan* plan, const double* param_dev, int coef_mode, double coef_scale,
                        double* inv_diag_dev, void* stream);

/* y = A x with the canonical CSR (FP64). Replaces LinearOperator.mv (solver_api.py:137-148). */
int femk_spmv(const femk_plan* plan, const double* vals_dev, const double* x_dev, double* y_dev,
              void* stream);

/* Gather CSR values into the solver's sliced-ELL copy held by the plan (32-row slices, column-major,
 * thread per row). femk_pcg does this itself at the start of every solve; this entry point and
 * femk_spmv_prepared expose the operator each PCG iteration multiplies with. No reference counterpart. */
int femk_prepare_operator(const femk_plan* plan, const double* vals_dev, void* stream);
int femk_spmv_prepared(const femk_plan* plan, const double* x_dev, double* y_dev, void* stream);

/* Opt-in CUDA-event timing of the FP64 CG loop's kernels (step SpMV, x/r/z update, p update),
 * accumulated over the iterations that ran since profiling was switched on. While it is on,
 * femk_pcg enqueues its chunks directly instead of replaying the chunk graph. */
int femk_set_profiling(femk_plan* plan, int on);
int femk_get_profile(const femk_plan* plan, double* step_ms, double* update_ms, double* pupdate_ms,
                     int64_t* iterations);

/* y = A x without an assembled matrix: per-element K_e x_e from coordinates and k_e. */
int femk_spmv_matfree(const femk_plan* plan, const double* param_dev, int coef_mode,
                      double coef_scale, const double* x_dev, double* y_dev, void* stream);

/*
 * Jacobi-preconditioned CG with jax.scipy.sparse.linalg.cg semantics (jNO: jno.solve.cg,
 * jno/solve.py:191-206). x_dev holds x0 on entry (zeros for jax's default) and the solution on
 * exit. inv_diag_dev may be NULL (no preconditioner). Stops when <r, r> <= max(tol^2 <b,b>, atol^2)
 * (<r, z> without a preconditioner) or after maxiter iterations. iters_out / relres_out may be
 * NULL; relres is ||b - A x|| / (||b|| + 1e-30) of the returned x (the eager guard of
 * solver_api.py:224-240). matfree_param_dev != NULL selects the matrix-free operator (vals_dev
 * is then ignored and may be NULL; inv_diag_dev must come from an assembled diagonal).
 */
int femk_pcg(const femk_plan* plan, const double* vals_dev, const double* b_dev, double* x_dev,
             const double* inv_diag_dev, double tol, double atol, int32_t maxiter, int32_t* iters_out,
             double* relres_out, void* stream);

int femk_pcg_matfree(const femk_plan* plan, const double* param_dev, int coef_mode, double coef_scale,
                     const double* b_dev, double* x_dev, const double* inv_diag_dev, double tol,
                     double atol, int32_t maxiter, int32_t* iters_out, double* relres_out, void* stream);

/*
 * Jacobi-preconditioned BiCGStab with jax.scipy.sparse.linalg.bicgstab semantics (jax 0.10.1):
 * stop when <r, r> <= max(tol^2 <b, b>, atol^2) or after maxiter iterations; a breakdown
 * (<rhat, r> = 0, alpha = 0 or omega = 0) ends the loop with x as it stands and returns
 * FEMK_BREAKDOWN. x holds x0 on entry and the solution on return; inv_diag may be NULL (no
 * preconditioner). *iters_out = iterations run, *relres_out = ||b - A x|| / (||b|| + 1e-30).
 * Replaces jno.solve.bicgstab (jno/solve.py:209-213) and the steady fem.solve() default
 * (jno/_fem.py:110-116, Jacobi-BiCGStab).
 */
int femk_bicgstab(const femk_plan* plan, const double* vals_dev, const double* b_dev, double* x_dev,
                  const double* inv_diag_dev, double tol, double atol, int32_t maxiter, int32_t* iters_out,
                  double* relres_out, void* stream);

/*
 * Restarted GMRES with jax.scipy.sparse.linalg.gmres semantics (jax 0.10.1, solve_method="batched"):
 * restart cycles of m = min(restart, n) Arnoldi steps (one classical Gram-Schmidt pass, the least
 * squares by Cholesky of its normal equations), stopping when ||M (b - A x)|| <= ||M b||
 * min(1, max(tol ||b||, atol) / ||b||) after a cycle, or after maxiter cycles (maxiter < 0: jax's
 * default 10 n; 0: no cycle). M = diag(inv_diag_dev), or the identity when NULL. x holds x0 on entry and the
 * solution on return. 1 <= restart <= 64. *iters_out = Arnoldi steps, *cycles_out = restart cycles,
 * *relres_out = ||b - A x|| / (||b|| + 1e-30) (each may be NULL). Returns FEMK_NOT_CONVERGED after
 * maxiter cycles (x written). The Krylov basis is plan-owned ((restart + 3) vectors, allocated on
 * first use). Replaces jno.solve.gmres (jno/solve.py:216-221); the theta march's step rescue
 * (femk_theta_march) runs the same iteration.
 */
int femk_gmres(const femk_plan* plan, const double* vals_dev, const double* b_dev, double* x_dev,
               const double* inv_diag_dev, double tol, double atol, int32_t restart, int64_t maxiter,
               int32_t* iters_out, int32_t* cycles_out, double* relres_out, void* stream);

/*
 * Consistent mass matrix M[a][b] = integral(phi_a phi_b) in the canonical CSR (vals_dev f64[nnz]).
 * zero_dirichlet != 0 leaves the Dirichlet rows and columns at zero, the transient block's M
 * (bcoo_zero_rows_cols, jno/utils/solver/fem_1d.py:939-949). Replaces the mass jacobian of the
 * temporal terms (jno/utils/solver/fem_native.py:2846-2850).
 */
int femk_mass_matrix(const femk_plan* plan, int zero_dirichlet, double* vals_dev, void* stream);

/*
 * Theta-step operators of the linear first-order block M u' + A u = c + f, assembled once on the
 * canonical CSR pattern (replaces the transient assembly of jno/utils/solver/fem_native.py:2846-3110
 * and the step-operator composition _add_step_operator, jno/utils/solver/solver_api.py:856-878):
 *   step_vals f64[nnz] = M' + theta dt A'        (the system of every step)
 *   rhs_vals  f64[nnz] = M' - (1 - theta) dt A'  (rhs = rhs_vals u + q, backend_blocks.py:342)
 *   q         f64[n]   = dt (c' + f')
 * M' is the consistent mass with Dirichlet rows and columns zeroed. A' is the stiffness of
 * k grad u . grad v (coefficient as in femk_assemble), with Dirichlet rows set to identity rows:
 *   FEMK_DIRICHLET_SYMMETRIC: Dirichlet columns eliminated, c' = load - A e lift, c'[d] = g[d]
 *     (_apply_dirichlet_transient, fem_1d.py:939-949: the route of a form without runtime parameters);
 *   FEMK_DIRICHLET_ROWS: Dirichlet columns kept, c'[d] = g[d] and f' = the load on free rows
 *     (bcoo_set_dirichlet_rows + the free-mask forcing, fem_native.py:3058-3087: the parametric route).
 * g f64[n] or NULL (0). 0 < theta <= 1 (1 backward Euler, 1/2 Crank-Nicolson); dt > 0.
 */
int femk_assemble_theta(const femk_plan* plan, const double* param_dev, int coef_mode, double scale, double f,
                        const double* g_dev, double theta, double dt, int dirichlet, double* step_vals_dev,
                        double* rhs_vals_dev, double* q_dev, void* stream);

/*
 * nsteps theta steps of the linear block (SemidiscreteTimeBlock.step, backend_blocks.py:332-413):
 *   rhs = rhs_vals u + q;  u <- Jacobi-BiCGStab(step_vals, rhs, x0 = u, tol, atol = 0, maxiter)
 * with the Jacobi inverse of diag(step_vals) (|d| <= 1e-30 -> 1), jax bicgstab semantics as
 * femk_bicgstab. After each step the relative residual ||S u - rhs|| / max(||rhs||, eps) must be
 * below step_check: 1e-9 is the reference's check of its default step solve (tol 1e-10). A step
 * that fails it, or whose BiCGStab stopped on its cap, a breakdown or a non-finite value, is
 * re-solved from x0 = the previous state by the GMRES of femk_gmres with tol = 1e-10, atol = 0,
 * restart = min(n, 40), the same Jacobi M and jax's default cap of 10 n restart cycles
 * (backend_blocks.py:402-413); the march stops with FEMK_NOT_CONVERGED only if that GMRES does not
 * converge. step_check <= 0 skips the check, as the solver-slot path of
 * compose_transient_step_solvers (jno/utils/solver/solver_api.py:929-945) does; BiCGStab's status
 * then stands. u_dev f64[n] holds the state (in/out); traj_dev f64[nsteps*n] or NULL receives the
 * state after every step; iters_out i32[nsteps] (host) or NULL: BiCGStab iterations per step;
 * gmres_out i32[nsteps] (host) or NULL: the rescue's Arnoldi steps per step (0 when the check
 * held); *relres_out (host, may be NULL) = the largest BiCGStab step residual. The step operator is
 * gathered into the plan's solver layout once per call: it replaces the operator a previous
 * femk_prepare_operator left there (femk_spmv_prepared then applies S until the next prepare).
 */
int femk_theta_march(const femk_plan* plan, const double* step_vals_dev, const double* rhs_vals_dev,
                     const double* q_dev, double* u_dev, int32_t nsteps, double tol, int32_t maxiter,
                     double step_check, double* traj_dev, int32_t* iters_out, int32_t* gmres_out,
                     double* relres_out, void* stream);

/*
 * Allocation-free Jacobi-PCG: the same iteration and result as femk_pcg, for callers that must
 * not allocate device memory during the call -- an XLA FFI handler (device memory is owned by XLA's
 * allocator), a framework whose caching allocator already holds nearly all of HBM, or a real-time
 * loop with a fixed memory budget. The plan (built once at set-up) and the caller's vectors are
 * the only other memory used; it calls no cudaMalloc/cudaFree and no allocating library routine.
 * Its workspace is one file-scope device array sized for FEMK_NOALLOC_MAX_N DOFs (about 8.5 MB),
 * which every GPU that loads the library holds until the process exits. Larger systems are
 * rejected with FEMK_EINVAL. The first call on a device looks up that array's device address
 * (cudaGetSymbolAddress) with the plan's device current; make that first call before any stream
 * capture. All calls share the array, so calls that overlap on the GPU (two streams, two
 * threads) race and must be serialised by the caller. No counterpart in the reference.
 */
#define FEMK_NOALLOC_MAX_N 262144
int femk_pcg_noalloc(const femk_plan* plan, const double* vals_dev, const double* b_dev, double* x_dev,
                     const double* inv_diag_dev, double tol, double atol, int32_t maxiter, int32_t* iters_out,
                     double* relres_out, void* stream);

/*
 * Mixed precision: inner CG on FP32 values and vectors, FP64 outer residual b - A x with the FP64
 * values and an FP64 solution. Converges to the same stopping rule as femk_pcg (on the true FP64
 * residual). mode = FEMK_MIXED_*. inner_iters_out counts FP32 iterations, outer_out FP64
 * residual evaluations. No reference counterpart (jNO runs x64 throughout).
 */
int femk_pcg_mixed(const femk_plan* plan, const double* vals_dev, const double* b_dev, double* x_dev,
                   const double* inv_diag_dev, double tol, double atol, int32_t maxiter, int mode,
                   int32_t* inner_iters_out, int32_t* outer_out, double* relres_out, void* stream);

/*
 * Batched Jacobi-PCG: nprob independent systems held by one plan built on their disjoint union
 * (vertex ids offset per problem), problem k owning rows [row_off[k], row_off[k+1]) (host array,
 * row_off[0] = 0, row_off[nprob] = n). One persistent cooperative launch runs every problem's CG
 * (jax cg semantics, per-problem alpha/beta/stop test) until all have stopped; rows are processed
 * in warp tiles of tile_rows (never crossing a problem) with blocks_per_sm (1 or 2) blocks of 16
 * warps per SM -- the schedule an autotuner chooses. iters_out / relres_out / status_out are host arrays of nprob
 * (may be NULL). Returns the first non-OK problem status, FEMK_TIMEOUT if a grid barrier gave up.
 * No reference counterpart (jNO batches by vmap over right-hand sides only).
 */
int femk_pcg_batched(const femk_plan* plan, int32_t nprob, const int64_t* row_off_host, const double* vals_dev,
                     const double* b_dev, double* x_dev, const double* inv_diag_dev, double tol, double atol,
                     int32_t maxiter, int32_t tile_rows, int32_t blocks_per_sm, int32_t* iters_out_host,
                     double* relres_out_host, int32_t* status_out_host, void* stream);

/*
 * femk_pcg_batched in mixed precision: FP32 values (converted from vals_dev in the same graph)
 * and FP32 inner vectors with FP32 SpMV accumulation, x in FP64, and per-problem FP64 reliable
 * updates (r = fp32(b - A x) with the FP64 values once the FP32 <r, r> fell by 1e-4 since the last
 * update, met the stop test or hit the cap; the direction is kept), as femk_pcg_mixed does for one
 * problem. Problem k retires when its FP64 <r, r> <= max(tol^2 <b, b>, atol^2) or at maxiter FP32
 * iterations. iters_out_host = FP32 iterations, outer_out_host = FP64 residual evaluations (may be
 * NULL); the other arguments as femk_pcg_batched (inv_diag_dev may be NULL: no preconditioner).
 * On plans with int16 column offsets and rows of at most 16 entries (P1 tetrahedra) and with
 * tile_rows <= 512 the launch uses 92-96 KB of dynamic shared memory a block (a two-stage ring a
 * warp that streams the FP32 slices and the update-phase operands). No reference counterpart.
 */
int femk_pcg_batched_mixed(const femk_plan* plan, int32_t nprob, const int64_t* row_off_host, const double* vals_dev,
                           const double* b_dev, double* x_dev, const double* inv_diag_dev, double tol, double atol,
                           int32_t maxiter, int32_t tile_rows, int32_t blocks_per_sm, int32_t* iters_out_host,
                           int32_t* outer_out_host, double* relres_out_host, int32_t* status_out_host, void* stream);

/*
 * Adjoint contraction: grad[c] = -k_c * (m o lam)_e^T K_hat_e (m o u)_e, m = 1 - dirichlet mask,
 * k_c = coef_scale * exp(param_c) (FEMK_COEF_EXP) or coef_scale (FEMK_COEF_LINEAR: d/dparam).
 * Nodal P1 modes: grad f64[nvert], grad[i] = sum over elements e holding vertex i of
 * -(m o lam)_e^T K_hat_e (m o u)_e * dk_e/dparam_i.
 * Replaces jax.grad through custom_linear_solve + segment_sum + jacfwd (no jNO function).
 */
int femk_adjoint_grad(const femk_plan* plan, const double* param_dev, int coef_mode, double coef_scale,
                      const double* u_dev, const double* lam_dev, double* grad_dev, void* stream);

/* Lumped mass m_i = sum over elements of integral(phi_i) (= the unit-source load before Dirichlet). */
int femk_lumped_mass(const femk_plan* plan, double* mass_dev, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FEMK_H */
