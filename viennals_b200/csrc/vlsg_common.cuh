// vlsg_common.cuh -- device data layout and helpers of libvlsgpu.
//
// Layout in HBM (per context):
//   * brick map: dense int32 array over a box of 8^3-cell bricks covering the
//     domain (bounded directions) or the band plus a margin (infinite
//     directions).  Entry >= 0: slot of an allocated brick; -1: not allocated.
//   * per level-set buffer and brick: int8 sign of an unallocated brick
//     (every cell undefined with that sign).
//   * slot pool: per buffer one value array of slots x 512 cells (x fastest,
//     then y, then z inside a brick) holding the value in grid units or
//     +-max for undefined cells, updated in place, and per slot a 512-bit
//     mask of the defined cells (8 words, one per z-plane, bit y*8+x).
//   * slot list: compact list of allocated slots, slot -> brick index, and
//     per slot its 27 neighbours (slot, or -1-brick when not allocated).
// Undefined cells carry the reference's sentinels +-numeric_limits<T>::max()
// (lsDomain.hpp:51-52) so every rule compares exactly as the reference does.
#pragma once

#include <cfloat>
#include <climits>
#include <cstdint>

#include "../../include/vlsg.h"

namespace vlsg {

constexpr int BS = 8;           // brick edge
constexpr int BV = BS * BS * BS; // cells per brick
constexpr int MAXB = 2 * VLSG_MAX_LEVEL_SETS; // current + initial copies

template <class T> struct Lim;
template <> struct Lim<double> {
  static __host__ __device__ constexpr double max() { return DBL_MAX; }
  static __host__ __device__ constexpr double lowest() { return -DBL_MAX; }
  static __host__ __device__ constexpr double eps() { return DBL_EPSILON; }
};
template <> struct Lim<float> {
  static __host__ __device__ constexpr float max() { return FLT_MAX; }
  static __host__ __device__ constexpr float lowest() { return -FLT_MAX; }
  static __host__ __device__ constexpr float eps() { return FLT_EPSILON; }
};

template <class T> __host__ __device__ inline bool isDef(T v) {
  return v != Lim<T>::max() && v != Lim<T>::lowest();
}

// Batching form: several independent domains share one brick box, stacked
// in z (each in its own range of brick planes, so that every domain's HRLE
// order is one contiguous stretch of the box's).  Per domain: its brick
// extent in x and y (the periodic extent / 8; it starts at the box's first
// brick) and its brick planes [bz0, bz1).  Every domain is periodic in x and
// y with extents that are multiples of the brick edge and unbounded in z, so
// no cell of the box is remapped: the 27-neighbour table wraps whole bricks
// within each domain.
struct DomainDev {
  int nbx, nby;
  int bz0, bz1;
};

// Grid and brick-map geometry, passed by value to kernels.
struct GridDev {
  int gmin[3], gmax[3]; // index bounds of the grid
  int bc[3];            // vlsg_boundary
  int org[3];           // global cell index of brick (0,0,0), cell (0,0,0)
  int nb[3];            // bricks per direction in the map box
  double delta;
  // batching form (nDom > 0): the domains and the domain of every brick plane
  int nDom;
  const DomainDev *dom;
  const int *domOfBz;
  // D = 2: the plane z = 0 of a grid periodic in z with period 1, so every
  // z neighbour of a cell is the cell itself and every z difference is 0
  int planar;
};

__host__ __device__ inline int mapCoord(const GridDev &g, int d, int c) {
  const int lo = g.gmin[d], hi = g.gmax[d];
  switch (g.bc[d]) {
  case VLSG_PERIODIC_BOUNDARY: {
    const int n = hi - lo;
    if (c >= lo && c < hi) return c;
    int r = (c - lo) % n;
    if (r < 0) r += n;
    return lo + r;
  }
  case VLSG_REFLECTIVE_BOUNDARY:
    for (int k = 0; k < 4; ++k) {
      if (c < lo) c = 2 * lo - c;
      else if (c > hi) c = 2 * hi - c;
      else break;
    }
    return c;
  case VLSG_POS_INFINITE_BOUNDARY:
    return c < lo ? 2 * lo - c : c;
  case VLSG_NEG_INFINITE_BOUNDARY:
    return c > hi ? 2 * hi - c : c;
  default:
    return c;
  }
}

// Buffer view: one level set (a current one or an RK initial copy).
template <class T> struct Buf {
  const T *vals;          // slot pool values
  const int8_t *farSign;  // per-brick sign of unallocated bricks
};

struct MapView {
  const int *brickMap;  // brick -> slot or -1
  const int *slotBrick; // slot -> linear brick index
};

__device__ inline int brickIndex(const GridDev &g, int bx, int by, int bz) {
  return (bz * g.nb[1] + by) * g.nb[0] + bx;
}

// Batching form: brick (x, y, z) next to a brick of domain d (x, y at most
// one brick outside d's extent), wrapped in x and y within d; false when z
// lies outside d's brick planes.
__device__ inline bool domainNeighbour(const GridDev &g, int d, int &x, int &y, int &z) {
  const DomainDev D = g.dom[d];
  x = (x + D.nbx) % D.nbx;
  y = (y + D.nby) % D.nby;
  return z >= D.bz0 && z < D.bz1;
}

// Value of global cell (x,y,z) (already mapped through the boundary
// conditions).  Cells outside the map box take the value of the nearest box
// cell: the box keeps a margin of undefined bricks around every band.
template <class T>
__device__ inline T cellValue(const GridDev &g, const MapView &m, const Buf<T> &b,
                              int x, int y, int z) {
  int rx = x - g.org[0], ry = y - g.org[1], rz = z - g.org[2];
  const int ex = g.nb[0] * BS - 1, ey = g.nb[1] * BS - 1, ez = g.nb[2] * BS - 1;
  rx = rx < 0 ? 0 : (rx > ex ? ex : rx);
  ry = ry < 0 ? 0 : (ry > ey ? ey : ry);
  rz = rz < 0 ? 0 : (rz > ez ? ez : rz);
  const int bi = brickIndex(g, rx >> 3, ry >> 3, rz >> 3);
  const int slot = m.brickMap[bi];
  if (slot < 0) return b.farSign[bi] < 0 ? Lim<T>::lowest() : Lim<T>::max();
  return b.vals[(size_t)slot * BV + ((rz & 7) * 64 + (ry & 7) * 8 + (rx & 7))];
}

// Pool index (slot * 512 + cell) of mapped cell (x,y,z), with cellValue's
// clamping; only for a cell whose value is defined (its brick has a slot).
__device__ inline size_t cellIndex(const GridDev &g, const MapView &m, int x, int y, int z) {
  int rx = x - g.org[0], ry = y - g.org[1], rz = z - g.org[2];
  const int ex = g.nb[0] * BS - 1, ey = g.nb[1] * BS - 1, ez = g.nb[2] * BS - 1;
  rx = rx < 0 ? 0 : (rx > ex ? ex : rx);
  ry = ry < 0 ? 0 : (ry > ey ? ey : ry);
  rz = rz < 0 ? 0 : (rz > ez ? ez : rz);
  const int slot = m.brickMap[brickIndex(g, rx >> 3, ry >> 3, rz >> 3)];
  return (size_t)slot * BV + ((rz & 7) * 64 + (ry & 7) * 8 + (rx & 7));
}

template <class T>
__device__ inline T cellValueRaw(const GridDev &g, const MapView &m,
                                 const Buf<T> &b, int x, int y, int z) {
  return cellValue<T>(g, m, b, mapCoord(g, 0, x), mapCoord(g, 1, y),
                      mapCoord(g, 2, z));
}

// hi + lo of a value with a compensation term; a zero term leaves hi as it is
// (keeping the sign of a zero).
__host__ __device__ inline double withLo(double hi, float lo) {
  return lo != 0.f ? hi + (double)lo : hi;
}

// cellValueRaw as a double, plus the compensation term `lo` of a defined
// value when the buffer carries one (lo non-null).
template <class T>
__device__ inline double cellValueFull(const GridDev &g, const MapView &m, const Buf<T> &b,
                                       const float *lo, int x, int y, int z) {
  x = mapCoord(g, 0, x), y = mapCoord(g, 1, y), z = mapCoord(g, 2, z);
  const T v = cellValue<T>(g, m, b, x, y, z);
  double r = (double)v;
  if (lo && isDef(v)) r = withLo(r, lo[cellIndex(g, m, x, y, z)]);
  return r;
}

__device__ inline void brickCoords(const GridDev &g, int bi, int &bx, int &by,
                                   int &bz) {
  bx = bi % g.nb[0];
  const int t = bi / g.nb[0];
  by = t % g.nb[1];
  bz = t / g.nb[1];
}

// A cell that exists in the grid (bounded directions have a fixed number of
// points; the last brick of a direction may hang over the end).
__device__ inline bool cellExists(const GridDev &g, int x, int y, int z) {
  const int c[3] = {x, y, z};
  for (int d = 0; d < 3; ++d) {
    if (g.bc[d] == VLSG_PERIODIC_BOUNDARY && (c[d] < g.gmin[d] || c[d] >= g.gmax[d]))
      return false;
    if (g.bc[d] == VLSG_REFLECTIVE_BOUNDARY && (c[d] < g.gmin[d] || c[d] > g.gmax[d]))
      return false;
    if (g.bc[d] == VLSG_POS_INFINITE_BOUNDARY && c[d] < g.gmin[d]) return false;
    if (g.bc[d] == VLSG_NEG_INFINITE_BOUNDARY && c[d] > g.gmax[d]) return false;
  }
  return true;
}

// Order-preserving 64-bit image of a non-negative double, for atomicMin/Max.
__device__ inline unsigned long long orderedBits(double v) {
  return (unsigned long long)__double_as_longlong(v);
}

} // namespace vlsg
