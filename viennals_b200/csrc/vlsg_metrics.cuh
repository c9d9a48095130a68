// vlsg_metrics.cuh -- comparison of two level sets on the device, for the
// precision report of the FP32 path against the FP64 path:
//   * point sets: defined and active (|phi| <= 0.5) points present in one
//     level set only, max / RMS |phi_a - phi_b| over the common points;
//   * volume: cells whose 8-corner average is <= 0 (the inside rule of
//     lsCompareVolume.hpp:272-287), over the map box;
//   * Chamfer distance between the zero-crossing node sets: a node on every
//     grid edge between two defined points of opposite sign, placed as
//     lsToSurfaceMesh.hpp:339-361 interpolates it (no merging of nodes closer
//     than the reference's minimum node distance), nearest neighbours found
//     exactly by searching grid cells in growing Chebyshev shells
//     (lsCompareChamfer.hpp:148-242 reports the same means / RMS / max).
// This header holds the per-engine parts (volume, nodes); the comparison of
// the two point / node sets is in vlsg_compare.cuh.  Both level sets are
// read through their exchange arrays (points in HRLE order, values as
// double), so they may have different storage types.
#pragma once

#include "vlsg_common.cuh"
#include "vlsg_exchange.cuh"

namespace vlsg {
namespace { // internal linkage: every compilation unit has its own copy

// Cells of the map box whose corner average is <= 0 (one warp per brick; a
// brick whose own and +x/+y/+z neighbour bricks are all unallocated with one
// sign is decided at once).
template <class T>
__global__ void kInsideCells(GridDev g, MapView m, Buf<T> b, int nBricks,
                             unsigned long long *count, const float *lo) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nWarps = (gridDim.x * blockDim.x) >> 5;
  unsigned long long inside = 0;
  for (int bi = warp; bi < nBricks; bi += nWarps) {
    int bx, by, bz;
    brickCoords(g, bi, bx, by, bz);
    // uniform test over the brick and the 7 bricks its +1 corners reach
    int sgn = 0;
    bool uniform = true;
    for (int k = 0; k < 8 && uniform; ++k) {
      int x = bx + (k & 1), y = by + ((k >> 1) & 1), z = bz + (k >> 2);
      x = x < g.nb[0] ? x : g.nb[0] - 1;
      y = y < g.nb[1] ? y : g.nb[1] - 1;
      z = z < g.nb[2] ? z : g.nb[2] - 1;
      const int nb = brickIndex(g, x, y, z);
      if (m.brickMap[nb] >= 0) uniform = false;
      else {
        const int s = b.farSign[nb] < 0 ? -1 : 1;
        if (sgn == 0) sgn = s;
        else if (s != sgn) uniform = false;
      }
    }
    if (uniform && g.bc[0] != VLSG_REFLECTIVE_BOUNDARY && g.bc[1] != VLSG_REFLECTIVE_BOUNDARY &&
        g.bc[2] != VLSG_REFLECTIVE_BOUNDARY && g.bc[0] != VLSG_PERIODIC_BOUNDARY &&
        g.bc[1] != VLSG_PERIODIC_BOUNDARY && g.bc[2] != VLSG_PERIODIC_BOUNDARY) {
      if (lane == 0 && sgn < 0) inside += BV;
      continue;
    }
    const int x0 = g.org[0] + bx * BS, y0 = g.org[1] + by * BS, z0 = g.org[2] + bz * BS;
    for (int c = lane; c < BV; c += 32) {
      const int x = x0 + (c & 7), y = y0 + ((c >> 3) & 7), z = z0 + (c >> 6);
      if (!cellExists(g, x, y, z)) continue;
      double sum = 0;
      for (int k = 0; k < 8; ++k)
        sum += cellValueFull<T>(g, m, b, lo, x + (k & 1), y + ((k >> 1) & 1), z + (k >> 2));
      inside += (sum / 8.0 <= 0.0) ? 1 : 0;
    }
  }
  for (int o = 16; o > 0; o >>= 1) inside += __shfl_xor_sync(0xffffffffu, inside, o);
  if (lane == 0 && inside) atomicAdd(count, inside);
}

// Zero-crossing nodes of the +x/+y/+z edges of every point: count pass
// (nodes == nullptr) or write pass at the scanned offsets.
template <class T>
__global__ void kSurfaceNodes(GridDev g, MapView m, Buf<T> b, const int32_t *idx,
                              const double *val, int64_t n, uint32_t *cnt, const uint32_t *off,
                              double *nodes, uint64_t *nodeKeys, const float *lo) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    const int c[3] = {idx[3 * p], idx[3 * p + 1], idx[3 * p + 2]};
    const double d0 = val[p];
    uint32_t k = 0, o = nodes ? off[p] : 0;
    for (int dir = 0; dir < 3; ++dir) {
      const T v1 = cellValueRaw<T>(g, m, b, c[0] + (dir == 0), c[1] + (dir == 1), c[2] + (dir == 2));
      if (!isDef(v1)) continue;
      const double d1 =
          cellValueFull<T>(g, m, b, lo, c[0] + (dir == 0), c[1] + (dir == 1), c[2] + (dir == 2));
      if ((d0 >= 0.) == (d1 >= 0.)) continue;
      if (nodes) {
        double pos[3] = {(double)c[0], (double)c[1], (double)c[2]};
        double cc;
        if (d0 == -d1) cc = c[dir] + 0.5;
        else if (fabs(d0) <= fabs(d1)) cc = c[dir] + (d0 / (d0 - d1));
        else cc = (c[dir] + 1) - (d1 / (d1 - d0));
        cc = fmax(cc, c[dir] + 1e-12);
        cc = fmin(cc, (c[dir] + 1) - 1e-12);
        pos[dir] = cc;
        for (int z = 0; z < 3; ++z) nodes[3 * (size_t)(o + k) + z] = pos[z];
        nodeKeys[o + k] = cellKey(c[0], c[1], c[2]);
      }
      ++k;
    }
    if (!nodes) cnt[p] = k;
  }
}

} // namespace
} // namespace vlsg
