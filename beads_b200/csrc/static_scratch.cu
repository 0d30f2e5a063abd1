// static_scratch.cu -- cell binning + stable counting sort that allocates
// nothing.
//
// Some callers cannot call cudaMalloc: a host code that owns every byte of
// device memory through its own pool, or a step loop that must not
// synchronize the device (cudaMalloc and cudaFree synchronize implicitly).
// For them this file keeps the per-cell counters in a file-scope device array
// of fixed size, kStaticMaxCells entries each for counts and cursors
// (2 x 65,536 x 4 B = 512 KiB, held by every GPU that loads the library until
// the process exits).  The caller passes the positions and the output arrays.
//
// The algorithm is the engine's rebuild front end (cell id from
// (x - lo) * inv_cell with the same clamp, counts, exclusive scan, scatter,
// ascending order inside every cell), written here as its own kernels so the
// engine's code paths stay untouched.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "../../include/beads_b200.h"
#include "setup.hpp"

namespace bb {
// Defined with the rest of the C ABI (capi.cpp): records the message that
// beads_last_error() returns on this thread.
void set_last_error(const char* message);
namespace {

constexpr uint32_t kStaticMaxCells = BEADS_STATIC_MAX_CELLS;
constexpr int kStaticThreads = 256;
constexpr int kStaticScanThreads = 1024;

// Shared by every call on a device; contents survive from the previous call.
static __device__ __align__(256) uint32_t g_static_scratch[2 * kStaticMaxCells];

__device__ __forceinline__ uint32_t static_axis_cell(float x, float lo, float inv, uint32_t n) {
  const float scaled = __fmul_rn(__fsub_rn(x, lo), inv);
  if (scaled <= 0.0f) return 0u;
  if (scaled >= (float)n) return n - 1u;
  const uint32_t idx = (uint32_t)scaled;
  return idx >= n ? n - 1u : idx;
}

struct StaticGrid {
  float lo[3];
  float inv_cell[3];
  uint32_t nc[3];
  uint32_t n_cells;
};

__global__ void k_static_clear(uint32_t* counts, uint32_t n_cells) {
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n_cells;
       c += gridDim.x * blockDim.x) {
    counts[c] = 0u;
  }
}

__global__ void k_static_bin(const float* pos, uint32_t n, StaticGrid g, uint32_t* cell_of,
                             uint32_t* counts) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t ix = static_axis_cell(pos[3 * (size_t)i], g.lo[0], g.inv_cell[0], g.nc[0]);
  const uint32_t iy = static_axis_cell(pos[3 * (size_t)i + 1], g.lo[1], g.inv_cell[1], g.nc[1]);
  const uint32_t iz = static_axis_cell(pos[3 * (size_t)i + 2], g.lo[2], g.inv_cell[2], g.nc[2]);
  const uint32_t cell = ix + g.nc[0] * (iy + g.nc[1] * iz);
  cell_of[i] = cell;
  atomicAdd(&counts[cell], 1u);
}

// One block: exclusive scan of the counts into cell_start (n_cells + 1
// entries) and the scatter cursors.
__global__ void __launch_bounds__(kStaticScanThreads)
k_static_scan(const uint32_t* counts, uint32_t* cursor, uint32_t* cell_start, uint32_t n_cells,
              uint32_t n) {
  __shared__ uint32_t sums[kStaticScanThreads];
  const uint32_t per = (n_cells + kStaticScanThreads - 1) / kStaticScanThreads;
  const uint32_t begin = min(n_cells, threadIdx.x * per);
  const uint32_t end = min(n_cells, begin + per);
  uint32_t local = 0;
  for (uint32_t c = begin; c < end; ++c) local += counts[c];
  sums[threadIdx.x] = local;
  __syncthreads();
  for (int o = 1; o < kStaticScanThreads; o <<= 1) {
    const uint32_t add = threadIdx.x >= (uint32_t)o ? sums[threadIdx.x - o] : 0u;
    __syncthreads();
    sums[threadIdx.x] += add;
    __syncthreads();
  }
  uint32_t run = threadIdx.x > 0 ? sums[threadIdx.x - 1] : 0u;
  for (uint32_t c = begin; c < end; ++c) {
    cell_start[c] = run;
    cursor[c] = run;
    run += counts[c];
  }
  if (threadIdx.x == 0) cell_start[n_cells] = n;
}

__global__ void k_static_scatter(const uint32_t* cell_of, uint32_t n, uint32_t* cursor,
                                 uint32_t* order) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  order[atomicAdd(&cursor[cell_of[i]], 1u)] = i;
}

// Ascending particle index inside every cell.  Cells of up to 32 members:
// one warp each, a bitonic network in registers.  Larger cells: one block
// each (k_static_cellsort_big), so no cell is ever sorted by a single thread.
__global__ void k_static_cellsort(const uint32_t* cell_start, uint32_t n_cells, uint32_t* order) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t warps = blockDim.x / 32u;
  for (uint32_t c = blockIdx.x * warps + threadIdx.x / 32u; c < n_cells; c += gridDim.x * warps) {
    const uint32_t s0 = cell_start[c];
    const uint32_t s1 = cell_start[c + 1];
    const uint32_t m = s1 - s0;
    if (m <= 1u || m > 32u) continue;  // warp-uniform
    uint32_t val = lane < m ? order[s0 + lane] : 0xffffffffu;
    for (uint32_t k = 2; k <= 32; k <<= 1) {
      for (uint32_t j = k >> 1; j > 0; j >>= 1) {
        const uint32_t other = __shfl_xor_sync(0xffffffffu, val, j);
        const bool up = (lane & k) == 0u;
        const bool lower = (lane & j) == 0u;
        val = (lower == up) ? min(val, other) : max(val, other);
      }
    }
    if (lane < m) order[s0 + lane] = val;
  }
}

// Cells of more than 32 members, one block per cell at a time: an ascending
// bitonic network over the m members in place (the form without direction
// flips: the first exchange of a stage of width k pairs i with the mirror
// i ^ (k - 1), the later ones i with i ^ j; a partner at or past m stands
// for +infinity, so that exchange is skipped).  O(m log^2 m) compare-exchanges
// spread over the block, with a block barrier between passes; members are
// staged in shared memory when they fit, otherwise sorted where they lie.
constexpr uint32_t kStaticBigThreads = 1024;
constexpr uint32_t kStaticSmemKeys = 8192;  // 32 KiB of shared memory

__device__ __forceinline__ void static_exchange(uint32_t* a, uint32_t i, uint32_t partner,
                                                uint32_t m) {
  if (partner > i && partner < m) {
    const uint32_t x = a[i], y = a[partner];
    if (y < x) {
      a[i] = y;
      a[partner] = x;
    }
  }
}

__device__ void static_bitonic(uint32_t* a, uint32_t m) {
  for (uint32_t k = 2; k < 2u * m; k <<= 1) {
    for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
      static_exchange(a, i, i ^ (k - 1u), m);
    }
    __syncthreads();
    for (uint32_t j = k >> 2; j > 0; j >>= 1) {
      for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) static_exchange(a, i, i ^ j, m);
      __syncthreads();
    }
  }
}

__global__ void __launch_bounds__(kStaticBigThreads)
k_static_cellsort_big(const uint32_t* cell_start, uint32_t n_cells, uint32_t* order) {
  __shared__ uint32_t keys[kStaticSmemKeys];
  for (uint32_t c = blockIdx.x; c < n_cells; c += gridDim.x) {
    const uint32_t s0 = cell_start[c];
    const uint32_t m = cell_start[c + 1] - s0;
    if (m <= 32u) continue;  // block-uniform
    if (m <= kStaticSmemKeys) {
      for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) keys[i] = order[s0 + i];
      __syncthreads();
      static_bitonic(keys, m);
      for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) order[s0 + i] = keys[i];
    } else {
      static_bitonic(order + s0, m);
    }
    __syncthreads();
  }
}

int static_fail(int code, const char* message) {
  set_last_error(message);
  return code;
}

// Device address of the static array on the current device.  The host-side
// symbol is only a stand-in, never a device address; the address is looked up
// on every call (cheap), so a module reloaded after cudaDeviceReset is seen.
int scratch_for_current_device(uint32_t** out) {
  void* ptr = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&ptr, g_static_scratch);
  if (e != cudaSuccess || ptr == nullptr) {
    return static_fail(BEADS_ERR_CUDA,
                       "beads_cell_sort_static: cudaGetSymbolAddress of the static scratch "
                       "array failed.");
  }
  *out = static_cast<uint32_t*>(ptr);
  return BEADS_OK;
}

}  // namespace
}  // namespace bb

extern "C" int beads_cell_sort_static(const float* d_positions, uint32_t n, const float box_lo[3],
                                      const float box_hi[3], double cutoff, double skin,
                                      uint32_t* d_cell_of, uint32_t* d_order,
                                      uint32_t* d_cell_start, uint32_t cell_start_capacity,
                                      uint32_t* n_cells_out, void* stream) {
  using namespace bb;
  if (!d_positions || !d_cell_of || !d_order || !d_cell_start || !box_lo || !box_hi || n == 0) {
    return static_fail(BEADS_ERR_INVALID, "beads_cell_sort_static: NULL argument or n == 0.");
  }
  Plan plan;
  try {
    plan = make_plan(box_lo, box_hi, cutoff, skin);
  } catch (const std::exception& e) {
    return static_fail(BEADS_ERR_INVALID, e.what());
  }
  if (plan.n_cells > kStaticMaxCells) {
    return static_fail(BEADS_ERR_INVALID,
                       "beads_cell_sort_static: the cell grid exceeds BEADS_STATIC_MAX_CELLS "
                       "(65536); use the engine context instead.");
  }
  if (cell_start_capacity < plan.n_cells + 1) {
    return static_fail(BEADS_ERR_INVALID,
                       "beads_cell_sort_static: cell_start needs n_cells + 1 entries.");
  }
  uint32_t* scratch = nullptr;
  const int rc = scratch_for_current_device(&scratch);
  if (rc != BEADS_OK) return rc;
  uint32_t* counts = scratch;
  uint32_t* cursor = scratch + kStaticMaxCells;
  StaticGrid g;
  for (int a = 0; a < 3; ++a) {
    g.lo[a] = box_lo[a];
    g.inv_cell[a] = plan.inv_cell[a];
    g.nc[a] = plan.nc[a];
  }
  g.n_cells = plan.n_cells;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const uint32_t blocks = (n + kStaticThreads - 1) / kStaticThreads;
  // The counters keep the previous call's values: clear them first.
  k_static_clear<<<(plan.n_cells + kStaticThreads - 1) / kStaticThreads, kStaticThreads, 0, s>>>(
      counts, plan.n_cells);
  k_static_bin<<<blocks, kStaticThreads, 0, s>>>(d_positions, n, g, d_cell_of, counts);
  k_static_scan<<<1, kStaticScanThreads, 0, s>>>(counts, cursor, d_cell_start, plan.n_cells, n);
  k_static_scatter<<<blocks, kStaticThreads, 0, s>>>(d_cell_of, n, cursor, d_order);
  const uint32_t sort_blocks = (plan.n_cells + (kStaticThreads / 32) - 1) / (kStaticThreads / 32);
  k_static_cellsort<<<sort_blocks, kStaticThreads, 0, s>>>(d_cell_start, plan.n_cells, d_order);
  const uint32_t big_blocks = plan.n_cells < 592u ? plan.n_cells : 592u;  // 4 per SM at most
  k_static_cellsort_big<<<big_blocks, kStaticBigThreads, 0, s>>>(d_cell_start, plan.n_cells,
                                                                 d_order);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return static_fail(BEADS_ERR_CUDA, cudaGetErrorString(e));
  if (n_cells_out) *n_cells_out = plan.n_cells;
  return BEADS_OK;
}
