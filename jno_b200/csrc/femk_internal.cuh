// Internal declarations shared by the femk translation units (sm_100a only).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <string>

#include "../../include/femk.h"

#define FEMK_VERSION 10300

namespace femk {

constexpr int kWork32Vectors = 7;  // FP32 vectors of the mixed solvers (plan->work32 holds this many)

// Bounds-checked build (-DFEMK_BOUNDS_CHECK, jno_b200/libfemk_bounds.so): FEMK_IN_BOUNDS(i, n, err)
// is false when i lies outside [0, n), after recording FEMK_EBOUNDS in *err; the caller then skips
// the access, so a bad index becomes a returned status instead of a fault. In the normal build it is
// the constant true and generates no code.
#ifdef FEMK_BOUNDS_CHECK
constexpr bool kBoundsCheck = true;
__device__ __forceinline__ bool in_bounds(int64_t i, int64_t n, int* err) {
  if (i >= 0 && i < n) return true;
  if (err) atomicExch(err, FEMK_EBOUNDS);
  return false;
}
#define FEMK_IN_BOUNDS(i, n, err) ::femk::in_bounds((int64_t)(i), (int64_t)(n), (err))
#else
constexpr bool kBoundsCheck = false;
#define FEMK_IN_BOUNDS(i, n, err) true
#endif

// A gather functor with an index check in the bounds-checked build (the functor itself otherwise).
template <typename G>
struct Checked {
  G g;
  int64_t n;
  int* err;
  template <typename I>
  __device__ __forceinline__ auto operator()(I j) const -> decltype(g(j)) {
    if (!FEMK_IN_BOUNDS(j, n, err)) return decltype(g(j))(0);
    return g(j);
  }
};
template <typename G>
__device__ __forceinline__ auto checked(G g, int64_t n, int* err) {
  if constexpr (kBoundsCheck)
    return Checked<G>{g, n, err};
  else
    return g;
}

void set_error(const std::string& msg);
void clear_error();

// Every kernel launch of the library is written `k<<<counted_launch() + grid, ...>>>`: the call adds
// one to a process-wide counter (read by femk_kernel_launches) and returns 0.
int counted_launch();
// Launches made while a stream is being captured are not executions: capture brackets its
// recording with set_capturing(true/false) and each graph launch adds its kernel count.
void set_capturing(bool on);
void count_launches(int64_t k);

// Return FEMK_ECUDA with a message if a CUDA runtime call failed.
#define FEMK_CUDA_TRY(expr)                                                              \
  do {                                                                                   \
    cudaError_t _e = (expr);                                                             \
    if (_e != cudaSuccess) {                                                             \
      ::femk::set_error(std::string(#expr) + ": " + cudaGetErrorString(_e));           \
      return _e == cudaErrorMemoryAllocation ? FEMK_ENOMEM : FEMK_ECUDA;                \
    }                                                                                    \
  } while (0)

#define FEMK_CHECK_ARG(cond, msg)           \
  do {                                      \
    if (!(cond)) {                          \
      ::femk::set_error(msg);               \
      return FEMK_EINVAL;                   \
    }                                       \
  } while (0)

// A coefficient mode is valid for a plan: P0 modes anywhere, nodal P1 modes on P1 plans only;
// every mode but CONST reads param.
inline bool coef_mode_ok(const femk_plan* p, int mode, const double* param);

#define FEMK_TRY(expr)          \
  do {                          \
    int _s = (expr);            \
    if (_s != FEMK_OK) return _s; \
  } while (0)

// Runs the statement with the constant ND bound to a plan's local dof count: 3 / 6 = P1 / P2
// triangle, 4 / 10 = P1 / P2 tetrahedron.
#define FEMK_BY_ND(nd, ...)                \
  do {                                     \
    switch (nd) {                          \
      case 3: {                            \
        constexpr int ND = 3;              \
        __VA_ARGS__;                       \
      } break;                             \
      case 6: {                            \
        constexpr int ND = 6;              \
        __VA_ARGS__;                       \
      } break;                             \
      case 4: {                            \
        constexpr int ND = 4;              \
        __VA_ARGS__;                       \
      } break;                             \
      default: {                           \
        constexpr int ND = 10;             \
        __VA_ARGS__;                       \
      } break;                             \
    }                                      \
  } while (0)

// Device-side solver scalars of one CG run. Lives in plan-owned device memory.
struct CgState {
  double gamma;     // <r, z>
  double rr;        // <r, r>
  double pq;        // <p, A p>
  double alpha, beta;
  double atol2;     // max(tol^2 <b, b>, atol^2)
  double bb;        // <b, b>
  int32_t iter;     // iterations taken
  int32_t maxiter;
  int32_t done;     // 1 once the stop test holds (or on failure)
  int32_t status;   // FEMK_OK / FEMK_BREAKDOWN / FEMK_NONFINITE
  uint32_t ticket;  // last-block-done counter of the reduction in flight
  int32_t precond;  // 1 when inv_diag is used in the stop test (rs = <r, r>), 0: rs = gamma
  // mixed precision bookkeeping
  double rr_since;  // rr at the last reliable update
  int32_t inner;    // FP32 iterations
  int32_t outer;    // FP64 residual evaluations
  int32_t xpend;    // split update: 1 while x += alpha p of the current iteration is still to be applied
};

}  // namespace femk

struct femk_plan {
  int device = 0;
  int order = 1, nd = 4;
  int dim = 3, nv = 4;  // spatial dimension, vertices per element (triangles: 2, 3)
  int64_t ntet = 0, nvert = 0, n = 0, nnz = 0, n_dir = 0;  // ntet: elements (tetrahedra or triangles)
  // pattern (plan-owned device memory)
  double* xyz = nullptr;        // f64[nvert*3] P1 vertex coordinates (z = 0 in 2-D)
  double* points = nullptr;     // f64[n*3] DOF coordinates
  int32_t* cells = nullptr;     // i32[ntet*nd]
  int32_t* indptr = nullptr;    // i32[n+1]
  int32_t* indices = nullptr;   // i32[nnz]
  int32_t* slot = nullptr;      // i32[ntet*nd*nd]
  int32_t* diag = nullptr;      // i32[n]
  uint8_t* dmask = nullptr;     // u8[n]
  int32_t* dlist = nullptr;     // i32[n_dir] ascending
  int32_t* inc_ptr = nullptr;   // i32[n+1] DOF -> element incidence
  int32_t* inc_elem = nullptr;  // i32[ntet*nd]
  int16_t* cols16 = nullptr;    // i16[nnz] col - row, when every entry fits
  int max_row = 0;              // longest CSR row
  int asm_rows = 128;           // rows per block of the row-gather assembly
  int64_t asm_span = 0;         // largest CSR span (entries) of asm_rows consecutive rows
  int* dev_err = nullptr;       // device error word of kernels whose index checks can only fail on a corrupt plan
  // assembly stream (femk_plan.cu, build_assembly_stream): per (free row, incident element) pair in
  // 32-row slices, the element, its unit-coefficient stiffness row (nd planes) and column positions
  int64_t* astr_ptr = nullptr;  // i64[n_slices+1] first entry of each slice
  int64_t astr_len = 0;         // entries (padding included)
  int32_t* astr_elem = nullptr; // i32[astr_len] element, -1 = padding
  double* astr_k = nullptr;     // f64[nd * astr_len] K_hat[a][c], plane c
  uint8_t* astr_pos = nullptr;  // u8[astr_len * pb] column positions in the row (0xff: Dirichlet column), pb = nd rounded up to 4
  double* astr_load = nullptr;  // f64[n] integral of the row's basis function (0 on Dirichlet rows)
  int spmv_L = 16, spmv_U = 2;  // SpMV lanes per row / rows in flight per lane group
  // sliced-ELL solver layout (SELL-32), built with the pattern
  int64_t n_slices = 0, sell_nnz = 0;
  int64_t* sell_ptr = nullptr;   // i64[n_slices+1] first entry of each slice
  int32_t* sell_cols = nullptr;  // i32[sell_nnz]
  int16_t* sell_c16 = nullptr;   // i16[sell_nnz] col - row, when the bandwidth fits
  double* sell_vals = nullptr;   // f64[sell_nnz] values gathered for the current solve
  float* sell_vals32 = nullptr;  // f32[sell_nnz] FP32 values for the mixed-precision inner solve
  // per-slice column tables of the bulk-copy SpMV (int16 offsets): a slice whose rows share one
  // offset sequence stores it once (padded to 8), any other slice its 32*w per-entry offsets
  int sell_uni = 1;
  int64_t* sell_cuptr = nullptr;  // i64[n_slices+1] first table entry of each slice
  int16_t* sell_cu = nullptr;     // i16[sell_cu_len]
  int64_t sell_cu_len = 0;
  int use_sell = 1;
  int l2_mode = 0;               // L2 eviction hints of the FP64 CG kernels (the l2_hints plan option)
  int sell64_c16 = 1;            // FP64 sliced-ELL streams int16 column offsets when available
  int sell_batch = 16;           // entries in flight per thread of the thread-per-row FP64 sliced-ELL kernel
                                 // (16: 16 with int16 columns, 32 with int32 columns)
  double mixed_delta2 = 0.0;     // reliable-update threshold of the mixed solvers (0: 1e-4)
  long long barrier_spin = 0;    // clock64 budget of each grid-barrier wait of the batched solvers
  int skip_arrival = -1;         // testing: block that skips its first grid-barrier arrival (-1: none)
  // solver workspace (allocated on first use)
  int64_t vstride = 0;          // solver vector stride: n rounded up to 64 (keeps every slot 512-byte aligned)
  double* work = nullptr;       // 5 slots of vstride doubles: r, z, p, q, p' (double-buffered direction)
  double* partials = nullptr;   // reduction partials
  femk::CgState* state = nullptr;
  femk::CgState* state_host = nullptr;  // pinned mirror
  float* work32 = nullptr;      // kWork32Vectors FP32 vectors of the mixed solvers
  float* vals32 = nullptr;      // FP32 copy of the values (mixed precision)
  double* work64b = nullptr;    // mixed-precision solver state
  int n_sm = 148;
  // CG launch machinery: plan-owned stream, events, and the captured chunk graph
  int cg_graph = 1;
  int cg_split = 1;             // split vector kernels (k_update_r + k_pupdate_x) on aligned vectors
  int bulk_cfg = 0;             // bulk-copy FP64 CG-step SpMV: 10 * stages + warps per block, 0 = off
  int bulk32_cfg = 0;           // the same for the FP32 step of the mixed solver
  int vec_blocks = 0;           // blocks per SM of the CG vector kernels (0: one full wave)
  int coop = 0;                 // device supports cooperative launch
  void* bar = nullptr;          // grid barrier of the batched solvers
  cudaStream_t cg_stream = nullptr;
  cudaEvent_t cg_ev[3] = {nullptr, nullptr, nullptr};
  cudaGraphExec_t cg_exec = nullptr;
  const void* cg_key[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  int cg_nodes = 0;
  // the same for the mixed-precision solver
  cudaStream_t mx_stream = nullptr;
  cudaEvent_t mx_ev[3] = {nullptr, nullptr, nullptr};
  cudaGraphExec_t mx_exec = nullptr;
  const void* mx_key[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  int mx_nodes = 0;
  void* mx_host = nullptr;  // pinned state mirrors
  // batched solver workspace (tiles, per-problem state, partials)
  void* batch_ws = nullptr;
  int64_t batch_bytes = 0;
  const void* batch_key[8] = {};
  cudaGraphExec_t batch_exec = nullptr;
  cudaStream_t batch_stream = nullptr;
  cudaEvent_t batch_ev = nullptr;
  int batch_graph_ok = 1;
  void* prof = nullptr;         // per-kernel CG timing (femk_set_profiling)
  double* coef_tmp = nullptr;   // f64[ntet] element coefficients of a nodal parameter
  double* kcoef = nullptr;      // f64[ntet] exp(param) of the current assembly or matrix-free solve
  int32_t* mcells = nullptr;    // i32[ntet*nd] cells with each Dirichlet DOF d as -1 - d (matrix-free operator)
  int32_t* kuhn = nullptr;      // i32[ntet/6*8] masked corners of each Kuhn block (P1 matrix-free, hex at a time)
  int kuhn_state = 0;           // 0 not checked, 1 every block of six tets is a Kuhn block, -1 not
  double* theta_ws = nullptr;   // f64[3 vstride] theta march: step Jacobi inverse, step right-hand side, previous state
  double* gm_ws = nullptr;      // GMRES: Krylov basis (restart + 1 vectors), w, q, partials, small arrays
  int64_t gm_size = 0;          // doubles in gm_ws
  int64_t* cmp_ws = nullptr;    // i64[2 n + 2] femk_compact: kept entries per row, then their exclusive scan
  // BiCGStab workspace (8 vectors), state, stream, events and captured chunk graph
  void* bicg_ws = nullptr;
  void* bicg_state = nullptr;
  void* bicg_host = nullptr;
  cudaStream_t bicg_stream = nullptr;
  cudaEvent_t bicg_ev[3] = {nullptr, nullptr, nullptr};
  cudaGraphExec_t bicg_exec = nullptr;
  const void* bicg_key[2] = {nullptr, nullptr};
  int batch_graph_used = 0;
};

namespace femk {

inline bool coef_mode_ok(const femk_plan* p, int mode, const double* param) {
  if (mode < FEMK_COEF_EXP || mode > FEMK_COEF_NODAL_LINEAR) return false;
  if (mode >= FEMK_COEF_NODAL_EXP && p->order != 1) return false;
  return mode == FEMK_COEF_CONST || param != nullptr;
}

// grid-size helpers
inline int blocks_for(int64_t n, int threads, int cap = 1 << 30) {
  int64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return (int)b;
}

// In the bounds-checked build: wait for `s`, read and clear the plan's device error word, and
// return FEMK_EBOUNDS (message naming `what`) if a kernel recorded a failed index check. In the
// normal build: FEMK_OK without touching the device.
int check_bounds(const femk_plan* p, cudaStream_t s, const char* what);

// Exclusive scan of int64 values: out[0..n] with out[n] = total. Works in place only when
// in != out is false-safe (it is not: pass distinct buffers).
int scan_exclusive_i64(const int64_t* in, int64_t* out, int64_t n, cudaStream_t s);

int ensure_workspace(femk_plan* p);

// The sliced-ELL value copies of a caller's CSR values (femk_cg.cu): ensure_sell_values allocates
// sell_vals (and, fp32, sell_vals32) and sets the copy kernels' shared-memory size (not during a
// graph capture); launch_sell_values enqueues the copies (FP64, and the unscaled FP32 values).
int ensure_sell_values(femk_plan* p, bool fp32);
int launch_sell_values(const femk_plan* p, const double* vals, bool fp32, cudaStream_t s);

// Nodal P1 coefficient modes become a per-element coefficient (plan-owned f64[ntet], computed on
// stream s) read as FEMK_COEF_LINEAR; other modes pass through unchanged.
int resolve_coef(const femk_plan* p, const double* param, int mode, cudaStream_t s, const double** param_out,
                 int* mode_out);
// resolve_coef, then FEMK_COEF_EXP as well: exp(param) once per element into the plan's kcoef
// buffer, read as FEMK_COEF_LINEAR (callers that visit an element more than once per call)
int resolve_coef_exp(const femk_plan* p, const double* param, int mode, cudaStream_t s, const double** param_out,
                     int* mode_out);

// Restarted GMRES (femk_gmres.cu) on the plan's prepared sliced-ELL operator (sell) or the canonical
// CSR values; x holds x0 on entry and the solution on return.
struct GmresInfo {
  int64_t steps = 0, cycles = 0;  // Arnoldi steps, restart cycles
  double beta = 0.0;              // final ||M (b - A x)||
  double rr = 0.0, bb = 0.0;      // final ||b - A x||^2 and ||b||^2
};
int gmres_run(femk_plan* p, bool sell, const double* vals, const double* b, double* x, const double* dinv,
              double tol, double atol, int restart, int64_t maxiter, cudaStream_t s, GmresInfo* info);

// Blocks of `threads` threads of kernel `fn` resident per SM (occupancy), cached per kernel.
int resident_blocks(const void* fn, int threads);

// One full wave of a grid-stride kernel: SMs x resident blocks (at most 8 per SM, which the
// reduction partial buffers are sized for).
template <typename K>
inline int wave_grid(K kernel, int threads, const femk_plan* p) {
  const int b = resident_blocks((const void*)kernel, threads);
  return p->n_sm * (b < 8 ? b : 8);
}

// Grid of the CG vector kernels: one wave, or p->vec_blocks blocks per SM when set (fewer blocks
// mean fewer partials for the last-block reduction to add).
template <typename K>
inline int vec_grid(K kernel, int threads, const femk_plan* p) {
  const int w = wave_grid(kernel, threads, p);
  return p->vec_blocks > 0 ? std::min(w, p->n_sm * p->vec_blocks) : w;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace femk
