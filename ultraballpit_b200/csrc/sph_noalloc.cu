// sph_noalloc.cu - neighbour-grid build that allocates no device memory.
//
// For callers that cannot call cudaMalloc: host engines that own every byte
// of device memory through their own pool or budget and forbid libraries
// from allocating, and callers on latency-critical paths where cudaMalloc or
// cudaFree would synchronize the device and stall their other streams. The
// caller passes device input and output arrays; the only scratch (per-cell
// cursors, scan tile sums, an error word) lives in the file-scope array
// g_grid_scratch below, which every GPU that loads this library holds until
// the process exits (2 MiB + 1 KiB).
//
// Output is NeighborGrid::update (kernel/src/neighbor.rs:82-122) in the
// reference's linear cell layout: per particle its cell hash, per cell the
// count and exclusive-scan offset, and the particle indices grouped by cell
// in ascending index (the reference's stable scatter).
#include <cstdint>
#include <mutex>

#include <cuda_runtime.h>

#include "sph_cuda.h"

namespace {

constexpr uint32_t kMaxCells = SPH_NOALLOC_MAX_CELLS;
constexpr uint32_t kTile = 2048;                  // cells per scan tile
constexpr uint32_t kMaxTiles = kMaxCells / kTile;  // 256
constexpr int kMaxPerCell = 1024;                  // particles per cell
constexpr int kSortWarps = 8;
constexpr int kScanThreads = 256;
constexpr int kScanPer = kTile / kScanThreads;  // 8

// [0, kMaxCells): per-cell write cursors; [kMaxCells, +kMaxTiles): scan tile
// sums; then one error word. Shared by every call on this device.
static __device__ __align__(256) uint32_t g_grid_scratch[kMaxCells + kMaxTiles + 64];

constexpr uint32_t kBsumOff = kMaxCells;
constexpr uint32_t kErrOff = kMaxCells + kMaxTiles;

std::mutex g_mu;
uint32_t* g_scratch_ptr[64] = {};  // device address of g_grid_scratch, per device

// Once per device, with that device current: the host-side name of the
// array is not a device address, so look the address up. *dev_out gets the
// current device.
int scratch_for_current_device(uint32_t** out, int* dev_out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return SPH_ERR_NO_DEVICE;
  *dev_out = dev;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_grid_scratch);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver ? SPH_ERR_NO_DEVICE : SPH_ERR_CUDA;
    }
    g_scratch_ptr[dev] = static_cast<uint32_t*>(p);
  }
  *out = g_scratch_ptr[dev];
  return SPH_OK;
}

struct GridGeom {
  float gmin[3];
  float cell;
  int dims[3];
};

// neighbor.rs:57-71: floor of the f32 quotient, clamped to the grid.
__device__ __forceinline__ int na_axis(float p, float gmin, float cell, int dim) {
  float f = floorf((p - gmin) / cell);
  f = fmaxf(f, 0.0f);
  f = fminf(f, (float)(dim - 1));
  return (int)f;
}

// neighbor.rs:75-77
__device__ __forceinline__ int na_cell(float x, float y, float z, const GridGeom& g) {
  int cx = na_axis(x, g.gmin[0], g.cell, g.dims[0]);
  int cy = na_axis(y, g.gmin[1], g.cell, g.dims[1]);
  int cz = na_axis(z, g.gmin[2], g.cell, g.dims[2]);
  return cx + cy * g.dims[0] + cz * g.dims[0] * g.dims[1];
}

// Exclusive scan over the block's threads; *total gets the block sum.
__device__ __forceinline__ uint32_t na_block_scan(uint32_t v, uint32_t* total) {
  __shared__ uint32_t warp_sums[kScanThreads / 32];
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t x = v;
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[wid] = x;
  __syncthreads();
  if (wid == 0) {
    uint32_t s = lane < kScanThreads / 32 ? warp_sums[lane] : 0u;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < kScanThreads / 32) warp_sums[lane] = s;
  }
  __syncthreads();
  uint32_t before = wid > 0 ? warp_sums[wid - 1] : 0u;
  *total = warp_sums[kScanThreads / 32 - 1];
  __syncthreads();
  return before + x - v;
}

__global__ void k_na_clear(uint32_t* __restrict__ counts, uint32_t ncells, uint32_t* __restrict__ scratch) {
  uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < ncells) counts[c] = 0u;
  if (c == 0) scratch[kErrOff] = 0u;
}

__global__ void k_na_count(const float* __restrict__ x, const float* __restrict__ y,
                           const float* __restrict__ z, uint32_t n, GridGeom g,
                           uint32_t* __restrict__ cell_index, uint32_t* __restrict__ counts) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int c = na_cell(x[i], y[i], z[i], g);
  cell_index[i] = (uint32_t)c;
  atomicAdd(&counts[c], 1u);
}

__global__ void __launch_bounds__(kScanThreads)
k_na_tile_sums(const uint32_t* __restrict__ counts, uint32_t ncells, uint32_t* __restrict__ scratch) {
  uint32_t base = blockIdx.x * kTile + threadIdx.x * kScanPer;
  uint32_t s = 0;
  for (int j = 0; j < kScanPer; ++j)
    if (base + j < ncells) s += counts[base + j];
  uint32_t total;
  na_block_scan(s, &total);
  if (threadIdx.x == 0) scratch[kBsumOff + blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads)
k_na_scan_tiles(uint32_t ntiles, uint32_t* __restrict__ scratch) {
  uint32_t v = threadIdx.x < ntiles ? scratch[kBsumOff + threadIdx.x] : 0u;
  uint32_t total;
  uint32_t ex = na_block_scan(v, &total);
  if (threadIdx.x < ntiles) scratch[kBsumOff + threadIdx.x] = ex;
}

__global__ void __launch_bounds__(kScanThreads)
k_na_offsets(const uint32_t* __restrict__ counts, uint32_t ncells, uint32_t* __restrict__ offsets,
             uint32_t* __restrict__ scratch) {
  uint32_t base = blockIdx.x * kTile + threadIdx.x * kScanPer;
  uint32_t v[kScanPer];
  uint32_t s = 0;
  for (int j = 0; j < kScanPer; ++j) {
    v[j] = base + j < ncells ? counts[base + j] : 0u;
    s += v[j];
  }
  uint32_t total;
  uint32_t run = na_block_scan(s, &total) + scratch[kBsumOff + blockIdx.x];
  for (int j = 0; j < kScanPer; ++j) {
    if (base + j < ncells) {
      offsets[base + j] = run;
      scratch[base + j] = run;  // cursor
    }
    run += v[j];
  }
}

__global__ void k_na_fill(const uint32_t* __restrict__ cell_index, uint32_t n, uint32_t* __restrict__ sorted,
                          uint32_t* __restrict__ scratch) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t slot = atomicAdd(&scratch[cell_index[i]], 1u);
  sorted[slot] = i;
}

// One warp per cell: bitonic sort of the cell's indices in place, ascending.
__global__ void __launch_bounds__(kSortWarps * 32)
k_na_sort_cells(const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ counts, uint32_t ncells,
                uint32_t* __restrict__ sorted, uint32_t* __restrict__ scratch) {
  __shared__ uint32_t buf[kSortWarps][kMaxPerCell];
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t c = blockIdx.x * kSortWarps + warp;
  if (c >= ncells) return;
  uint32_t cnt = counts[c];
  if (cnt < 2) return;
  if (cnt > (uint32_t)kMaxPerCell) {
    if (lane == 0) atomicOr(&scratch[kErrOff], 1u);
    return;
  }
  uint32_t st = offsets[c];
  int m = 1;
  while (m < (int)cnt) m <<= 1;
  uint32_t* b = buf[warp];
  for (int q = lane; q < m; q += 32) b[q] = q < (int)cnt ? sorted[st + q] : 0xffffffffu;
  __syncwarp();
  for (int k = 2; k <= m; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int q = lane; q < m; q += 32) {
        int p = q ^ j;
        if (p > q) {
          uint32_t a = b[q], d = b[p];
          if ((a > d) == ((q & k) == 0)) { b[q] = d; b[p] = a; }
        }
      }
      __syncwarp();
    }
  }
  for (int q = lane; q < (int)cnt; q += 32) sorted[st + q] = b[q];
}

inline unsigned blocks(uint64_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

extern "C" int sph_grid_sort_noalloc(const float* d_x, const float* d_y, const float* d_z, uint32_t n,
                                     const float domain_min[3], const float domain_max[3], float cell_size,
                                     uint32_t* d_cell_index, uint32_t* d_cell_offsets,
                                     uint32_t* d_cell_counts, uint32_t* d_sorted, size_t cells_capacity,
                                     void* stream) {
  if (!domain_min || !domain_max || !(cell_size > 0.0f) || !d_cell_offsets || !d_cell_counts)
    return SPH_ERR_INVALID_ARG;
  if (n > 0 && (!d_x || !d_y || !d_z || !d_cell_index || !d_sorted)) return SPH_ERR_INVALID_ARG;
  if (n > 0x7fffffffu) return SPH_ERR_INVALID_ARG;
  GridGeom g;
  uint64_t ncells = 1;
  for (int a = 0; a < 3; ++a) {
    if (!(domain_max[a] > domain_min[a])) return SPH_ERR_INVALID_ARG;
    // neighbor.rs:31-35
    float d = fmaxf(ceilf((domain_max[a] - domain_min[a]) / cell_size), 1.0f);
    if (!(d <= (float)kMaxCells)) return SPH_ERR_CAPACITY;
    g.dims[a] = (int)d;
    g.gmin[a] = domain_min[a];
    ncells *= (uint64_t)g.dims[a];
  }
  g.cell = cell_size;
  if (ncells > kMaxCells) return SPH_ERR_CAPACITY;  // the scratch holds kMaxCells cursors
  if (ncells > cells_capacity) return SPH_ERR_INVALID_ARG;
  uint32_t C = (uint32_t)ncells;
  uint32_t* scratch = nullptr;
  int dev = 0;
  int s = scratch_for_current_device(&scratch, &dev);
  if (s != SPH_OK) return s;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // The scratch address belongs to the current device, and the call ends
  // with a host wait on the stream: a stream of another device, or one that
  // is capturing, is rejected before anything is enqueued.
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) {
    cudaGetLastError();
    return SPH_ERR_INVALID_ARG;
  }
  if (cap != cudaStreamCaptureStatusNone) return SPH_ERR_INVALID_ARG;
  if (st) {
    int sdev = -1;
    if (cudaStreamGetDevice(st, &sdev) != cudaSuccess) {
      cudaGetLastError();
      return SPH_ERR_INVALID_ARG;
    }
    if (sdev != dev) return SPH_ERR_INVALID_ARG;
  }
  uint32_t ntiles = (C + kTile - 1) / kTile;
  k_na_clear<<<blocks(C, 256), 256, 0, st>>>(d_cell_counts, C, scratch);
  if (n > 0) k_na_count<<<blocks(n, 256), 256, 0, st>>>(d_x, d_y, d_z, n, g, d_cell_index, d_cell_counts);
  k_na_tile_sums<<<ntiles, kScanThreads, 0, st>>>(d_cell_counts, C, scratch);
  k_na_scan_tiles<<<1, kScanThreads, 0, st>>>(ntiles, scratch);
  k_na_offsets<<<ntiles, kScanThreads, 0, st>>>(d_cell_counts, C, d_cell_offsets, scratch);
  if (n > 0) {
    k_na_fill<<<blocks(n, 256), 256, 0, st>>>(d_cell_index, n, d_sorted, scratch);
    k_na_sort_cells<<<blocks(C, kSortWarps), kSortWarps * 32, 0, st>>>(d_cell_offsets, d_cell_counts, C,
                                                                        d_sorted, scratch);
  }
  // a launch that failed leaves its outputs unwritten: report it here rather
  // than leave the error pending for the caller's next call
  if (cudaGetLastError() != cudaSuccess) return SPH_ERR_CUDA;
  uint32_t err = 0;
  cudaError_t e = cudaMemcpyAsync(&err, scratch + kErrOff, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return e == cudaErrorMemoryAllocation ? SPH_ERR_OOM : SPH_ERR_CUDA;
  return err ? SPH_ERR_CAPACITY : SPH_OK;
}
