// vlsg_voids.cuh -- setIgnoreVoids: MarkVoidPoints (lsMarkVoidPoints.hpp:
// 157-300) with its default options on the top level set, before the rates.
//
// The sign field (value >= 0 or < 0, :37-39) splits into star-connected
// components over the brick box.  Nodes: every cell of an allocated brick
// (slot * 512 + cell) and every unallocated brick as a whole (poolCells +
// brick: all its cells share the far sign).  A union-find over the nodes
// (lock-free linking of the larger root under the smaller, path halving)
// joins neighbours of the same sign through the boundary conditions.  The
// top component holds the box's last position in HRLE order (its last brick,
// last existing cell).  A defined point >= 0 is void when it lies outside the
// top component; a negative one when none of its star neighbours of the
// other sign lies in it (:268-287).  When the last position is negative
// nothing is marked.  The reference numbers HRLE runs rather than cells; the
// components of the two are the same sets of grid points.
#pragma once

#include "vlsg_common.cuh"

namespace vlsg {
namespace { // internal linkage: every compilation unit has its own copy

constexpr int VOID_ERR = 256; // union-find did not settle within its bound

__device__ inline uint32_t vFind(uint32_t *parent, uint32_t x, int *err) {
  for (int k = 0; k < (1 << 24); ++k) {
    const uint32_t p = parent[x];
    if (p == x) return x;
    const uint32_t gp = parent[p];
    if (gp != p) parent[x] = gp; // path halving (any interleaving keeps a valid forest)
    x = p;
  }
  atomicOr(err, VOID_ERR);
  return x;
}

__device__ inline void vUnite(uint32_t *parent, uint32_t a, uint32_t b, int *err) {
  for (int k = 0; k < (1 << 20); ++k) {
    a = vFind(parent, a, err);
    b = vFind(parent, b, err);
    if (a == b) return;
    if (a < b) {
      const uint32_t t = a;
      a = b;
      b = t;
    }
    if (atomicCAS(&parent[a], a, b) == a) return;
  }
  atomicOr(err, VOID_ERR);
}

// Node and value of global cell (x, y, z) after the boundary mapping; false
// when it lies outside the brick box (an infinite direction).
template <class T>
__device__ inline bool voidNode(const GridDev &g, const MapView &m, const Buf<T> &b,
                               size_t poolCells, int x, int y, int z, uint32_t &node, T &val) {
  x = mapCoord(g, 0, x), y = mapCoord(g, 1, y), z = mapCoord(g, 2, z);
  const int rx = x - g.org[0], ry = y - g.org[1], rz = z - g.org[2];
  if (rx < 0 || ry < 0 || rz < 0 || rx >= g.nb[0] * BS || ry >= g.nb[1] * BS || rz >= g.nb[2] * BS)
    return false;
  if (!cellExists(g, x, y, z)) return false;
  const int bi = brickIndex(g, rx >> 3, ry >> 3, rz >> 3);
  const int slot = m.brickMap[bi];
  if (slot < 0) {
    node = (uint32_t)(poolCells + bi);
    val = b.farSign[bi] < 0 ? Lim<T>::lowest() : Lim<T>::max();
  } else {
    const int c = (rz & 7) * 64 + (ry & 7) * 8 + (rx & 7);
    node = (uint32_t)((size_t)slot * BV + c);
    val = b.vals[(size_t)slot * BV + c];
  }
  return true;
}

__global__ void kVoidInit(uint32_t *parent, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    parent[i] = (uint32_t)i;
}

// Edges from every existing cell of the listed slots to its six neighbours.
template <class T>
__global__ void kVoidUnionCells(GridDev g, MapView m, Buf<T> b, const int *slotList,
                                const int *nSlots, size_t poolCells, uint32_t *parent, int *err) {
  const size_t n = (size_t)*nSlots * BV;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const int slot = slotList[i / BV], c = (int)(i % BV);
    int bx, by, bz;
    brickCoords(g, m.slotBrick[slot], bx, by, bz);
    const int x = g.org[0] + bx * BS + (c & 7), y = g.org[1] + by * BS + ((c >> 3) & 7),
              z = g.org[2] + bz * BS + (c >> 6);
    if (!cellExists(g, x, y, z)) continue;
    const uint32_t self = (uint32_t)((size_t)slot * BV + c);
    const bool pos = b.vals[(size_t)slot * BV + c] >= T(0);
    for (int j = 0; j < 6; ++j) {
      const int d = j % 3, s = j < 3 ? 1 : -1;
      uint32_t node;
      T val;
      if (!voidNode<T>(g, m, b, poolCells, x + (d == 0) * s, y + (d == 1) * s, z + (d == 2) * s,
                       node, val))
        continue;
      if ((val >= T(0)) == pos) vUnite(parent, self, node, err);
    }
  }
}

// Edges between face-adjacent unallocated bricks of the same far sign.
template <class T>
__global__ void kVoidUnionBricks(GridDev g, MapView m, Buf<T> b, int nBricks, size_t poolCells,
                                 uint32_t *parent, int *err) {
  for (int bi = blockIdx.x * blockDim.x + threadIdx.x; bi < nBricks; bi += gridDim.x * blockDim.x) {
    if (m.brickMap[bi] >= 0) continue;
    int bc[3];
    brickCoords(g, bi, bc[0], bc[1], bc[2]);
    for (int j = 0; j < 6; ++j) {
      const int d = j % 3, s = j < 3 ? 1 : -1;
      int nc[3] = {bc[0], bc[1], bc[2]};
      nc[d] += s;
      if (nc[d] < 0 || nc[d] >= g.nb[d]) {
        if (g.bc[d] != VLSG_PERIODIC_BOUNDARY) continue;
        nc[d] = (nc[d] + g.nb[d]) % g.nb[d];
      }
      const int bj = brickIndex(g, nc[0], nc[1], nc[2]);
      if (bj == bi || m.brickMap[bj] >= 0) continue;
      if ((b.farSign[bj] < 0) == (b.farSign[bi] < 0))
        vUnite(parent, (uint32_t)(poolCells + bi), (uint32_t)(poolCells + bj), err);
    }
  }
}

// top[0] = root of the box's last position, top[1] = 1 when it is >= 0.
template <class T>
__global__ void kVoidTop(GridDev g, MapView m, Buf<T> b, size_t poolCells, uint32_t *parent,
                         uint32_t *top, int *err) {
  if (blockIdx.x || threadIdx.x) return;
  top[0] = 0;
  top[1] = 0;
  const int x0 = g.org[0] + (g.nb[0] - 1) * BS, y0 = g.org[1] + (g.nb[1] - 1) * BS,
            z0 = g.org[2] + (g.nb[2] - 1) * BS;
  for (int c = BV - 1; c >= 0; --c) {
    const int x = x0 + (c & 7), y = y0 + ((c >> 3) & 7), z = z0 + (c >> 6);
    if (!cellExists(g, x, y, z)) continue;
    uint32_t node;
    T val;
    if (!voidNode<T>(g, m, b, poolCells, x, y, z, node, val)) continue;
    top[0] = vFind(parent, node, err);
    top[1] = val >= T(0) ? 1u : 0u;
    return;
  }
}

// Void bits of the defined cells of the listed slots (mask zeroed before).
template <class T>
__global__ void kVoidMark(GridDev g, MapView m, Buf<T> b, const int *slotList, const int *nSlots,
                          const uint64_t *def, size_t poolCells, uint32_t *parent,
                          const uint32_t *top, uint64_t *mask, int *err) {
  if (!top[1]) return;
  const uint32_t topRoot = top[0];
  const size_t n = (size_t)*nSlots * BV;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const int slot = slotList[i / BV], c = (int)(i % BV);
    if (!((def[(size_t)slot * 8 + (c >> 6)] >> (c & 63)) & 1ull)) continue;
    const T v = b.vals[(size_t)slot * BV + c];
    bool isVoid;
    if (v >= T(0)) {
      isVoid = vFind(parent, (uint32_t)((size_t)slot * BV + c), err) != topRoot;
    } else {
      int bx, by, bz;
      brickCoords(g, m.slotBrick[slot], bx, by, bz);
      const int x = g.org[0] + bx * BS + (c & 7), y = g.org[1] + by * BS + ((c >> 3) & 7),
                z = g.org[2] + bz * BS + (c >> 6);
      bool reached = false;
      for (int j = 0; j < 6 && !reached; ++j) {
        const int d = j % 3, s = j < 3 ? 1 : -1;
        uint32_t node;
        T val;
        if (!voidNode<T>(g, m, b, poolCells, x + (d == 0) * s, y + (d == 1) * s, z + (d == 2) * s,
                         node, val))
          continue;
        if (signbit(val) == signbit(v)) continue;
        reached = vFind(parent, node, err) == topRoot;
      }
      isVoid = !reached;
    }
    if (isVoid) atomicOr((unsigned long long *)&mask[(size_t)slot * 8 + (c >> 6)], 1ull << (c & 63));
  }
}

} // namespace
} // namespace vlsg
