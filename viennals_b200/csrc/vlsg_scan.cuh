// vlsg_scan.cuh -- exclusive prefix sums of uint32 arrays on the device
// (reduce, scan of the block sums, scan + offset), used to lay out the
// exchange format (points and undefined runs in HRLE order).
#pragma once

#include <cstdint>

namespace vlsg {
namespace { // internal linkage: every compilation unit has its own copy

constexpr int SCAN_THREADS = 512;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;     // elements per block
constexpr int SCAN_TOP_THREADS = 1024;
constexpr int SCAN_TOP_ITEMS = 32;
constexpr size_t SCAN_MAX = (size_t)SCAN_TILE * SCAN_TOP_THREADS * SCAN_TOP_ITEMS;

// Exclusive scan of one value per thread over the block; returns the block
// total in *total (every thread).
__device__ inline uint32_t blockExclusiveScan(uint32_t v, uint32_t *warpSums, uint32_t *total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  uint32_t x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += t;
  }
  if (lane == 31) warpSums[wid] = x;
  __syncthreads();
  if (wid == 0) {
    uint32_t s = lane < nw ? warpSums[lane] : 0u;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += t;
    }
    if (lane < nw) warpSums[lane] = s; // inclusive
  }
  __syncthreads();
  const uint32_t before = wid ? warpSums[wid - 1] : 0u;
  *total = warpSums[nw - 1];
  __syncthreads();
  return before + x - v;
}

__global__ void __launch_bounds__(SCAN_THREADS)
    kScanReduce(const uint32_t *in, size_t n, uint32_t *blockSums) {
  __shared__ uint32_t ws[32];
  const size_t base = (size_t)blockIdx.x * SCAN_TILE;
  uint32_t s = 0;
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    const size_t i = base + (size_t)k * SCAN_THREADS + threadIdx.x;
    if (i < n) s += in[i];
  }
  uint32_t total;
  blockExclusiveScan(s, ws, &total);
  if (threadIdx.x == 0) blockSums[blockIdx.x] = total;
}

// In place over the block sums (nb <= SCAN_TOP_THREADS * SCAN_TOP_ITEMS);
// the grand total lands in blockSums[nb].
__global__ void __launch_bounds__(SCAN_TOP_THREADS) kScanTop(uint32_t *blockSums, int nb) {
  __shared__ uint32_t ws[32];
  uint32_t v[SCAN_TOP_ITEMS];
  uint32_t s = 0;
  const int base = threadIdx.x * SCAN_TOP_ITEMS;
  for (int k = 0; k < SCAN_TOP_ITEMS; ++k) {
    v[k] = base + k < nb ? blockSums[base + k] : 0u;
    s += v[k];
  }
  uint32_t total;
  uint32_t off = blockExclusiveScan(s, ws, &total);
  for (int k = 0; k < SCAN_TOP_ITEMS; ++k) {
    if (base + k < nb) blockSums[base + k] = off;
    off += v[k];
  }
  if (threadIdx.x == 0) blockSums[nb] = total;
}

__global__ void __launch_bounds__(SCAN_THREADS)
    kScanApply(const uint32_t *in, size_t n, const uint32_t *blockOffsets, uint32_t *out) {
  __shared__ uint32_t tile[SCAN_TILE];
  __shared__ uint32_t ws[32];
  const size_t base = (size_t)blockIdx.x * SCAN_TILE;
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    const int j = k * SCAN_THREADS + threadIdx.x;
    tile[j] = base + j < n ? in[base + j] : 0u;
  }
  __syncthreads();
  uint32_t s = 0;
  for (int k = 0; k < SCAN_ITEMS; ++k) s += tile[threadIdx.x * SCAN_ITEMS + k];
  uint32_t total;
  uint32_t off = blockExclusiveScan(s, ws, &total) + blockOffsets[blockIdx.x];
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    const int j = threadIdx.x * SCAN_ITEMS + k;
    const uint32_t t = tile[j];
    tile[j] = off;
    off += t;
  }
  __syncthreads();
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    const int j = k * SCAN_THREADS + threadIdx.x;
    if (base + j < n) out[base + j] = tile[j];
  }
}

// Number of block sums (plus one for the total) a scan of n elements needs.
inline size_t scanScratch(size_t n) { return (n + SCAN_TILE - 1) / SCAN_TILE + 1; }

} // namespace
} // namespace vlsg
