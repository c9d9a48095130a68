// vlsg_maint.cuh -- slot-pool maintenance, upload and download kernels.
//
// After every stage the set of allocated bricks is brought back to "every
// brick holding a defined cell of any live level set, plus its 26
// neighbours": the band moves at most one cell per pass and at most a few
// cells between two maintenances, so every cell a pass can change lies in an
// allocated brick.  A freed brick records its (uniform) sign per level set in
// the far-sign map; a new brick starts with every cell undefined with that
// sign.
#pragma once

#include "vlsg_common.cuh"

namespace vlsg {
namespace { // internal linkage: every compilation unit has its own copy

struct BufSet {
  void *vals[MAXB];
  uint64_t *def[MAXB]; // current defined masks
  int8_t *farSign[MAXB];
  int nBuf;
};

__device__ inline bool slotHasDef(const uint64_t *def, int slot) {
  const uint64_t *w = def + (size_t)slot * 8;
  return (w[0] | w[1] | w[2] | w[3] | w[4] | w[5] | w[6] | w[7]) != 0ull;
}

__device__ inline bool neighbourBrick(const GridDev &g, int &x, int &y, int &z) {
  int c[3] = {x, y, z};
  for (int d = 0; d < 3; ++d) {
    if (c[d] < 0 || c[d] >= g.nb[d]) {
      if (g.bc[d] == VLSG_PERIODIC_BOUNDARY) c[d] = (c[d] + g.nb[d]) % g.nb[d];
      else return false; // reflective: mirrored cells lie inside the box
    }
  }
  x = c[0], y = c[1], z = c[2];
  return true;
}

__device__ inline void markDilated(const GridDev &g, int bi, uint8_t *needed, int *err) {
  int bx, by, bz;
  brickCoords(g, bi, bx, by, bz);
  if (g.nDom) {
    // the band must stay off the domain's first and last brick planes
    const int d = g.domOfBz[bz];
    if (bz <= g.dom[d].bz0 || bz >= g.dom[d].bz1 - 1) atomicOr(err, 1);
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          int x = bx + dx, y = by + dy, z = bz + dz;
          if (domainNeighbour(g, d, x, y, z)) needed[brickIndex(g, x, y, z)] = 1;
        }
    return;
  }
  const int c[3] = {bx, by, bz};
  for (int d = 0; d < 3; ++d)
    if (g.bc[d] != VLSG_PERIODIC_BOUNDARY && g.bc[d] != VLSG_REFLECTIVE_BOUNDARY &&
        (c[d] <= 0 || c[d] >= g.nb[d] - 1))
      atomicOr(err, 1);
  for (int dz = -1; dz <= 1; ++dz)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        int x = bx + dx, y = by + dy, z = bz + dz;
        if (neighbourBrick(g, x, y, z)) needed[brickIndex(g, x, y, z)] = 1;
      }
}

// err bits: 1 box too small (infinite direction), 4 pool capacity,
// 8 a freed brick still held a defined cell
__global__ void kMarkNeeded(GridDev g, const int *slotBrick, const int *slotList,
                            const int *nSlots, BufSet B, uint8_t *needed, int *err) {
  const int n = *nSlots;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int slot = slotList[i];
    bool core = false;
    for (int b = 0; b < B.nBuf; ++b) core |= slotHasDef(B.def[b], slot);
    if (core) markDilated(g, slotBrick[slot], needed, err);
  }
}

__global__ void kDilateBricks(GridDev g, int nBricks, const uint8_t *core,
                              uint8_t *needed, int *err) {
  for (int bi = blockIdx.x * blockDim.x + threadIdx.x; bi < nBricks;
       bi += gridDim.x * blockDim.x)
    if (core[bi]) markDilated(g, bi, needed, err);
}

// First cell of a brick that exists in the grid (cells of the last brick of
// a bounded direction may lie past its end).
__device__ inline int firstExistingCell(const GridDev &g, int bi) {
  int bx, by, bz;
  brickCoords(g, bi, bx, by, bz);
  const int x0 = g.org[0] + bx * BS, y0 = g.org[1] + by * BS, z0 = g.org[2] + bz * BS;
  for (int c = 0; c < BV; ++c)
    if (cellExists(g, x0 + (c & 7), y0 + ((c >> 3) & 7), z0 + (c >> 6))) return c;
  return 0;
}

template <class T>
__global__ void kFreeUnneeded(GridDev g, const int *slotList, const int *nSlots, int *brickMap,
                              int *slotBrick, const uint8_t *needed, BufSet B,
                              int *freeStack, int *freeCount, int *err) {
  const int n = *nSlots;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int slot = slotList[i];
    const int bi = slotBrick[slot];
    if (needed[bi]) continue;
    const int c = firstExistingCell(g, bi);
    for (int b = 0; b < B.nBuf; ++b) {
      if (slotHasDef(B.def[b], slot)) atomicOr(err, 8);
      const T v = ((const T *)B.vals[b])[(size_t)slot * BV + c];
      B.farSign[b][bi] = v < 0 ? -1 : 1;
    }
    brickMap[bi] = -1;
    slotBrick[slot] = -1;
    freeStack[atomicAdd(freeCount, 1)] = slot;
  }
}

// Allocate a slot for every needed brick without one; list the new slots.
__global__ void kAllocNeeded(int nBricks, int *brickMap, int *slotBrick, const uint8_t *needed,
                             int *freeStack, int *freeCount, int *newList, int *nNew,
                             int *err) {
  for (int bi = blockIdx.x * blockDim.x + threadIdx.x; bi < nBricks;
       bi += gridDim.x * blockDim.x) {
    if (!needed[bi] || brickMap[bi] >= 0) continue;
    const int k = atomicSub(freeCount, 1) - 1;
    if (k < 0) {
      atomicAdd(freeCount, 1);
      atomicOr(err, 4);
      continue;
    }
    const int slot = freeStack[k];
    brickMap[bi] = slot;
    slotBrick[slot] = bi;
    if (newList) newList[atomicAdd(nNew, 1)] = slot;
  }
}

// New slots are visited by the next pass: the face cells of their
// neighbours were not marked for them while they were unallocated.
struct VisitSet {
  uint8_t *p[MAXB];
  int n;
};
__global__ void kVisitNewSlots(const int *newList, const int *nNew, VisitSet v) {
  const int n = *nNew;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int slot = newList[i];
    for (int k = 0; k < v.n; ++k) v.p[k][slot] = 1;
  }
}

// New slots: every cell undefined with the brick's far sign, no defined cell.
// Cells past the end of a bounded direction hold +max.
template <class T>
__global__ void kInitNewSlots(GridDev g, const int *newList, const int *nNew,
                              const int *slotBrick, BufSet B) {
  const int n = *nNew;
  for (int it = blockIdx.x; it < n; it += gridDim.x) {
    const int slot = newList[it];
    const int bi = slotBrick[slot];
    int bx, by, bz;
    brickCoords(g, bi, bx, by, bz);
    for (int b = 0; b < B.nBuf; ++b) {
      const T s = B.farSign[b][bi] < 0 ? Lim<T>::lowest() : Lim<T>::max();
      T *v = (T *)B.vals[b] + (size_t)slot * BV;
      for (int c = threadIdx.x; c < BV; c += blockDim.x) {
        const bool ex = cellExists(g, g.org[0] + bx * BS + (c & 7),
                                   g.org[1] + by * BS + ((c >> 3) & 7), g.org[2] + bz * BS + (c >> 6));
        v[c] = ex ? s : Lim<T>::max();
      }
      if (threadIdx.x < 8) B.def[b][(size_t)slot * 8 + threadIdx.x] = 0ull;
    }
  }
}

// Slot list in brick order (warp-aggregated append).
__global__ void kBuildSlotList(int nBricks, const int *brickMap, int *slotList,
                               int *nSlots) {
  for (int base = blockIdx.x * blockDim.x; base < nBricks; base += gridDim.x * blockDim.x) {
    const int bi = base + threadIdx.x;
    const int slot = bi < nBricks ? brickMap[bi] : -1;
    const bool has = slot >= 0;
    const unsigned mask = __ballot_sync(0xffffffffu, has);
    const int lane = threadIdx.x & 31;
    int off = 0;
    if (lane == 0 && mask) off = atomicAdd(nSlots, __popc(mask));
    off = __shfl_sync(0xffffffffu, off, 0);
    if (has) slotList[off + __popc(mask & ((1u << lane) - 1))] = slot;
  }
}

__device__ inline uint64_t cellKey(int x, int y, int z) {
  const uint64_t off = 1ull << 20;
  return ((uint64_t)(z + (int)off) << 42) | ((uint64_t)(y + (int)off) << 21) |
         (uint64_t)(x + (int)off);
}

// Sign of the undefined run containing `key` (last run start <= key).
__device__ inline int8_t runSignAt(const uint64_t *keys, const int8_t *sign, int nRuns,
                                   uint64_t key) {
  if (nRuns <= 0) return 1;
  int lo = 0, hi = nRuns; // first index with keys[i] > key
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (keys[mid] <= key) lo = mid + 1;
    else hi = mid;
  }
  return lo == 0 ? sign[0] : sign[lo - 1];
}

// Far signs of all bricks of one brick row (by, bz) from the runs: the sign
// at each brick's centre cell; one binary search per row, then a walk along
// the row (the centre cells of a row have increasing keys).  Bounded
// directions map the centre cells (they lie inside the grid but for the
// last, partial brick, whose centre may be mapped).
__global__ void kFarSignRows(GridDev g, const uint64_t *runKeys, const int8_t *runSign, int nRuns,
                             int8_t *farSign) {
  const int rows = g.nb[1] * g.nb[2];
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
    const int by = r % g.nb[1], bz = r / g.nb[1];
    const int y = mapCoord(g, 1, g.org[1] + by * BS + 4), z = mapCoord(g, 2, g.org[2] + bz * BS + 4);
    int8_t *row = farSign + (size_t)r * g.nb[0];
    if (nRuns <= 0) {
      for (int bx = 0; bx < g.nb[0]; ++bx) row[bx] = 1;
      continue;
    }
    int j = -1, prevX = INT_MIN;
    for (int bx = 0; bx < g.nb[0]; ++bx) {
      const int x = mapCoord(g, 0, g.org[0] + bx * BS + 4);
      const uint64_t key = cellKey(x, y, z);
      if (x <= prevX || j < 0) { // first brick, or the mapping folded back: search
        int lo = 0, hi = nRuns;
        while (lo < hi) {
          const int mid = (lo + hi) >> 1;
          if (runKeys[mid] <= key) lo = mid + 1;
          else hi = mid;
        }
        j = lo - 1;
      } else {
        while (j + 1 < nRuns && runKeys[j + 1] <= key) ++j;
      }
      prevX = x;
      const int8_t s = j < 0 ? runSign[0] : runSign[j];
      row[bx] = s < 0 ? -1 : 1;
      if (j < 0) j = -1;
    }
  }
}

__global__ void kMarkPointBricks(GridDev g, int n, const int *idx, uint8_t *core,
                                 int *err) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int rx = idx[3 * i] - g.org[0], ry = idx[3 * i + 1] - g.org[1],
              rz = idx[3 * i + 2] - g.org[2];
    if (rx < 0 || ry < 0 || rz < 0 || rx >= g.nb[0] * BS || ry >= g.nb[1] * BS ||
        rz >= g.nb[2] * BS) {
      atomicOr(err, 1);
      continue;
    }
    core[brickIndex(g, rx >> 3, ry >> 3, rz >> 3)] = 1;
  }
}

// Undefined cells of every allocated brick from the runs' signs (before the
// points are scattered): one thread per x-row of a brick, one binary search
// per row and a walk along it; bricks next to a boundary that remaps cells
// look every cell up through the mapping.
template <class T>
__global__ void kFillRows(GridDev g, const int *slotList, const int *nSlots, const int *slotBrick,
                          const uint8_t *cflag, const uint64_t *keys, const int8_t *sign,
                          int nRuns, T *vals) {
  const size_t total = (size_t)*nSlots * 64;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    const int slot = slotList[e >> 6];
    const int lz = (int)(e >> 3) & 7, ly = (int)e & 7;
    int bx, by, bz;
    brickCoords(g, slotBrick[slot], bx, by, bz);
    const int x0 = g.org[0] + bx * BS, y = g.org[1] + by * BS + ly, z = g.org[2] + bz * BS + lz;
    T *row = vals + (size_t)slot * BV + lz * 64 + ly * 8;
    if (cflag[slot] & 1) { // CF_STAR
      for (int lx = 0; lx < 8; ++lx) {
        const int s = runSignAt(keys, sign, nRuns, cellKey(mapCoord(g, 0, x0 + lx), mapCoord(g, 1, y),
                                                           mapCoord(g, 2, z)));
        row[lx] = s < 0 ? Lim<T>::lowest() : Lim<T>::max();
      }
      continue;
    }
    if (nRuns <= 0) {
      for (int lx = 0; lx < 8; ++lx) row[lx] = Lim<T>::max();
      continue;
    }
    const uint64_t key0 = cellKey(x0, y, z);
    int lo = 0, hi = nRuns; // first run starting after key0
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (keys[mid] <= key0) lo = mid + 1;
      else hi = mid;
    }
    int j = lo - 1;
    for (int lx = 0; lx < 8; ++lx) {
      const uint64_t key = key0 + lx;
      while (j + 1 < nRuns && keys[j + 1] <= key) ++j;
      const int s = j < 0 ? sign[0] : sign[j];
      row[lx] = s < 0 ? Lim<T>::lowest() : Lim<T>::max();
    }
  }
}

// Uploaded points through the boundary mapping (in place), their index box
// (atomic min / max into box[0..5]) and the range check (err bit 128).
__global__ void kStagePoints(GridDev g, int n, int32_t *idx, int *box, int *err) {
  int mn[3] = {INT_MAX, INT_MAX, INT_MAX}, mx[3] = {INT_MIN, INT_MIN, INT_MIN};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    for (int d = 0; d < 3; ++d) {
      const int c = mapCoord(g, d, idx[3 * i + d]);
      if (c < -(1 << 19) || c > (1 << 19)) atomicOr(err, 128);
      idx[3 * i + d] = c;
      mn[d] = min(mn[d], c), mx[d] = max(mx[d], c);
    }
  }
  for (int d = 0; d < 3; ++d)
    for (int o = 16; o > 0; o >>= 1) {
      mn[d] = min(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], o));
      mx[d] = max(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], o));
    }
  if ((threadIdx.x & 31) == 0 && mn[0] != INT_MAX)
    for (int d = 0; d < 3; ++d) {
      atomicMin(&box[d], mn[d]);
      atomicMax(&box[3 + d], mx[d]);
    }
}

__device__ inline uint64_t runKey(const int32_t *start, int i) {
  int c[3];
  for (int d = 0; d < 3; ++d) {
    const int v = start[3 * i + d];
    c[d] = v < -(1 << 20) + 1 ? -(1 << 20) + 1 : (v > (1 << 20) - 1 ? (1 << 20) - 1 : v);
  }
  return cellKey(c[0], c[1], c[2]);
}

// HRLE keys of the run starts; *unsorted is set when they are out of order.
__global__ void kStageRuns(int n, const int32_t *start, uint64_t *keys, int *unsorted) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint64_t k = runKey(start, i);
    keys[i] = k;
    if (i > 0 && k < runKey(start, i - 1)) atomicOr(unsorted, 1);
  }
}

__global__ void kCountFlags(const uint8_t *f, int n, int *count) {
  for (int base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    const int i = base + threadIdx.x;
    const unsigned m = __ballot_sync(0xffffffffu, i < n && f[i]);
    if ((threadIdx.x & 31) == 0 && m) atomicAdd(count, __popc(m));
  }
}

__global__ void kInitFreeStack(int *freeStack, int cap) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cap; i += gridDim.x * blockDim.x)
    freeStack[i] = cap - 1 - i;
}

template <class T>
__global__ void kScatterPoints(GridDev g, int n, const int *idx, const double *v,
                               const int *brickMap, T *vals, int *err, float *lo) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int rx = idx[3 * i] - g.org[0], ry = idx[3 * i + 1] - g.org[1],
              rz = idx[3 * i + 2] - g.org[2];
    if (rx < 0 || ry < 0 || rz < 0 || rx >= g.nb[0] * BS || ry >= g.nb[1] * BS ||
        rz >= g.nb[2] * BS) {
      atomicOr(err, 1);
      continue;
    }
    const int slot = brickMap[brickIndex(g, rx >> 3, ry >> 3, rz >> 3)];
    if (slot < 0) {
      atomicOr(err, 4);
      continue;
    }
    const size_t q = (size_t)slot * BV + ((rz & 7) * 64 + (ry & 7) * 8 + (rx & 7));
    const T hi = T(v[i]);
    vals[q] = hi;
    // the part of the uploaded double that the storage type drops
    if (lo) lo[q] = (float)(v[i] - (double)hi);
  }
}


// Compensation terms of uploaded points: the part of each double that its
// float (already scattered) dropped.
template <class T>
__global__ void kScatterLo(GridDev g, int n, const int *idx, const double *v, const int *brickMap,
                           float *lo) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int rx = idx[3 * i] - g.org[0], ry = idx[3 * i + 1] - g.org[1],
              rz = idx[3 * i + 2] - g.org[2];
    if (rx < 0 || ry < 0 || rz < 0 || rx >= g.nb[0] * BS || ry >= g.nb[1] * BS ||
        rz >= g.nb[2] * BS)
      continue;
    const int slot = brickMap[brickIndex(g, rx >> 3, ry >> 3, rz >> 3)];
    if (slot < 0) continue;
    lo[(size_t)slot * BV + ((rz & 7) * 64 + (ry & 7) * 8 + (rx & 7))] =
        (float)(v[i] - (double)T(v[i]));
  }
}

// Defined masks and defined-cell count of a buffer from its values (after an
// upload); cells past the end of a bounded direction are set to +max.
template <class T>
__global__ void kMasksFromValues(GridDev g, const int *slotBrick, const int *slotList,
                                 const int *nSlots, T *vals, uint64_t *def,
                                 unsigned long long *cnt, unsigned long long *bound) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nWarps = (gridDim.x * blockDim.x) >> 5;
  const int n = *nSlots;
  double maxAbs = 0.0;
  for (int w = warp; w < n; w += nWarps) {
    const int slot = slotList[w];
    int bx, by, bz;
    brickCoords(g, slotBrick[slot], bx, by, bz);
    int nd = 0;
    uint64_t mine = 0;
    for (int z = 0; z < 8; ++z) {
      uint64_t bits = 0;
      for (int half = 0; half < 2; ++half) {
        const int c = z * 64 + half * 32 + lane;
        T v = vals[(size_t)slot * BV + c];
        if (!cellExists(g, g.org[0] + bx * BS + (c & 7), g.org[1] + by * BS + ((c >> 3) & 7),
                        g.org[2] + bz * BS + (c >> 6))) {
          v = Lim<T>::max();
          vals[(size_t)slot * BV + c] = v;
        }
        const unsigned m = __ballot_sync(0xffffffffu, isDef(v));
        bits |= (uint64_t)m << (32 * half);
        nd += lane == 0 ? __popc(m) : 0;
        if (isDef(v)) maxAbs = fmax(maxAbs, fabs((double)v));
      }
      if (lane == z) mine = bits;
    }
    if (lane < 8) def[(size_t)slot * 8 + lane] = mine;
    if (lane == 0 && nd && cnt) atomicAdd(cnt, (unsigned long long)nd);
  }
  if (bound) {
    for (int o = 16; o > 0; o >>= 1) maxAbs = fmax(maxAbs, __shfl_xor_sync(0xffffffffu, maxAbs, o));
    if (lane == 0 && maxAbs > 0.0) atomicMax(bound, (unsigned long long)__double_as_longlong(maxAbs));
  }
}

// `lo`: compensation terms of the buffer (or null), added to defined values.
template <class T>
__global__ void kQueryValues(GridDev g, MapView m, Buf<T> b, int n, const int *idx,
                             double *out, const float *lo) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int x = mapCoord(g, 0, idx[3 * i]), y = mapCoord(g, 1, idx[3 * i + 1]),
              z = mapCoord(g, 2, idx[3 * i + 2]);
    const T v = cellValue<T>(g, m, b, x, y, z);
    double r = isDef(v) ? (double)v : (v < 0 ? -DBL_MAX : DBL_MAX);
    if (lo && isDef(v)) r = withLo(r, lo[cellIndex(g, m, x, y, z)]);
    out[i] = r;
  }
}


// Defined cells of a buffer, from its masks.
__global__ void kCountDefined(const int *slotList, const int *nSlots, const uint64_t *def,
                              unsigned long long *cnt) {
  const int n = *nSlots;
  for (int base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    const int i = base + threadIdx.x;
    int nd = 0;
    if (i < n) {
      const uint64_t *w = def + (size_t)slotList[i] * 8;
      for (int k = 0; k < 8; ++k) nd += __popcll(w[k]);
    }
    for (int o = 16; o > 0; o >>= 1) nd += __shfl_xor_sync(0xffffffffu, nd, o);
    if ((threadIdx.x & 31) == 0 && nd) atomicAdd(cnt, (unsigned long long)nd);
  }
}

// Every cell of the listed slots set to v (undefined: v is a sentinel).
template <class T>
__global__ void kFillSlots(const int *slotList, const int *nSlots, T *vals, uint64_t *def, T v) {
  const size_t n = (size_t)*nSlots * BV;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const size_t slot = slotList[i / BV];
    vals[slot * BV + i % BV] = v;
    if (i % BV < 8) def[slot * 8 + i % BV] = 0ull;
  }
}

// BooleanOperation INVERT (lsBooleanOperation.hpp:215-255): every value of
// the listed slots negated (sentinels swap sign), and every far sign.
template <class T>
__global__ void kNegateSlots(const int *slotList, const int *nSlots, T *vals, int8_t *farSign,
                             int nBricks, float *lo) {
  const size_t n = (size_t)*nSlots * BV;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const size_t slot = slotList[i / BV];
    vals[slot * BV + i % BV] = -vals[slot * BV + i % BV];
    if (lo) lo[slot * BV + i % BV] = -lo[slot * BV + i % BV];
  }
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nBricks; b += gridDim.x * blockDim.x)
    farSign[b] = (int8_t)-farSign[b];
}

} // namespace
} // namespace vlsg
