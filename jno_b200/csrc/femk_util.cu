// Error reporting, version, and a device exclusive scan used by the plan build.
#include <algorithm>
#include <atomic>
#include <mutex>
#include <unordered_map>

#include "femk_internal.cuh"
#include "femk_spmv.cuh"

namespace femk {

static thread_local std::string g_last_error;
static std::atomic<int64_t> g_launches{0};

static thread_local bool g_capturing = false;

int counted_launch() {
  if (!g_capturing) g_launches.fetch_add(1, std::memory_order_relaxed);
  return 0;
}

void set_capturing(bool on) { g_capturing = on; }

void count_launches(int64_t k) { g_launches.fetch_add(k, std::memory_order_relaxed); }

void set_error(const std::string& msg) { g_last_error = msg; }

int resident_blocks(const void* fn, int threads) {
  static std::mutex mu;
  static std::unordered_map<const void*, int> cache;
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find(fn);
  if (it != cache.end()) return it->second;
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, threads, 0) != cudaSuccess || b < 1) b = 1;
  cache[fn] = b;
  return b;
}

void choose_spmv_cfg(double mean_row, int* L, int* U) {
  // measured on B200 at P1 128^3 (mean 14.8) and P2 64^3 (mean 28.4): 8 lanes x 2 rows in flight
  // beats 16x1/16x2/32x1/32x2 and 4x4, 8x4 by 20-60%
  if (mean_row <= 6.0) {
    *L = 4, *U = 4;
  } else if (mean_row <= 40.0) {
    *L = 8, *U = 2;
  } else {
    *L = 16, *U = 2;
  }
}
void clear_error() { g_last_error.clear(); }

}  // namespace femk

extern "C" int femk_bounds_checked(void) { return femk::kBoundsCheck ? 1 : 0; }

namespace femk {

int check_bounds(const femk_plan* p, cudaStream_t s, const char* what) {
  if (!kBoundsCheck) return FEMK_OK;
  int h = 0;
  FEMK_CUDA_TRY(cudaMemcpyAsync(&h, p->dev_err, sizeof(int), cudaMemcpyDeviceToHost, s));
  FEMK_CUDA_TRY(cudaStreamSynchronize(s));
  if (h == 0) return FEMK_OK;
  FEMK_CUDA_TRY(cudaMemsetAsync(p->dev_err, 0, sizeof(int), s));
  set_error(std::string(what) + ": an index check inside a kernel failed (bounds-checked build)");
  return FEMK_EBOUNDS;
}

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int64_t block_exclusive_scan(int64_t v, int64_t* total) {
  __shared__ int64_t warp_tot[kScanThreads / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int64_t inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int64_t t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) warp_tot[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    int64_t w = lane < kScanThreads / 32 ? warp_tot[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int64_t t = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += t;
    }
    if (lane < kScanThreads / 32) warp_tot[lane] = w;  // inclusive over warps
  }
  __syncthreads();
  int64_t before = wid > 0 ? warp_tot[wid - 1] : 0;
  *total = warp_tot[kScanThreads / 32 - 1];
  __syncthreads();
  return before + inc - v;
}

__global__ void k_tile_sums(const int64_t* __restrict__ in, int64_t n, int64_t* __restrict__ sums) {
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  int64_t s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i)
    if (base + i < n) s += in[base + i];
  __shared__ int64_t red[kScanThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    int64_t t = 0;
    for (int w = 0; w < kScanThreads / 32; ++w) t += red[w];
    sums[blockIdx.x] = t;
  }
}

__global__ void k_tile_scan(const int64_t* __restrict__ in, int64_t n, const int64_t* __restrict__ offs,
                            int64_t* __restrict__ out) {
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  int64_t v[kScanItems];
  int64_t s = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    v[i] = base + i < n ? in[base + i] : 0;
    s += v[i];
  }
  int64_t total;
  int64_t run = block_exclusive_scan(s, &total) + (offs ? offs[blockIdx.x] : 0);
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    if (base + i < n) out[base + i] = run;
    run += v[i];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = (offs ? offs[blockIdx.x] : 0) + total;
}

}  // namespace

int scan_exclusive_i64(const int64_t* in, int64_t* out, int64_t n, cudaStream_t s) {
  if (n <= 0) {
    FEMK_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(int64_t), s));
    return FEMK_OK;
  }
  const int64_t tiles = (n + kScanTile - 1) / kScanTile;
  if (tiles == 1) {
    k_tile_scan<<<::femk::counted_launch() + 1, kScanThreads, 0, s>>>(in, n, nullptr, out);
    FEMK_CUDA_TRY(cudaGetLastError());
    return FEMK_OK;
  }
  int64_t* sums = nullptr;
  int64_t* offs = nullptr;
  FEMK_CUDA_TRY(cudaMallocAsync(&sums, sizeof(int64_t) * tiles, s));
  FEMK_CUDA_TRY(cudaMallocAsync(&offs, sizeof(int64_t) * (tiles + 1), s));
  k_tile_sums<<<::femk::counted_launch() + (unsigned)tiles, kScanThreads, 0, s>>>(in, n, sums);
  FEMK_CUDA_TRY(cudaGetLastError());
  int st = scan_exclusive_i64(sums, offs, tiles, s);
  if (st == FEMK_OK) {
    k_tile_scan<<<::femk::counted_launch() + (unsigned)tiles, kScanThreads, 0, s>>>(in, n, offs, out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      set_error(std::string("scan: ") + cudaGetErrorString(e));
      st = FEMK_ECUDA;
    }
  }
  cudaFreeAsync(sums, s);
  cudaFreeAsync(offs, s);
  return st;
}

}  // namespace femk

extern "C" int femk_version(void) { return FEMK_VERSION; }

extern "C" int64_t femk_kernel_launches(void) { return femk::g_launches.load(std::memory_order_relaxed); }

extern "C" const char* femk_last_error_string(void) {
  static thread_local std::string copy;
  copy = femk::g_last_error;
  return copy.c_str();
}
