// vlsg_maint.cuh -- slot-pool maintenance, upload and download kernels.
//
// After every pass that can move the band, the set of allocated bricks is
// brought back to "every brick holding a defined cell of any live level set,
// plus its 26 neighbours": a band moves at most one cell per pass and at most
// a few cells between two maintenances, so reads never reach a brick whose
// cells are unknown.  A freed brick records its (uniform) sign per level set
// in the far-sign map; a new brick starts UNIFORM with that sign.
#pragma once

#include "vlsg_common.cuh"

namespace vlsg {

struct BufSet {
  const uint8_t *hasDef[MAXB];
  uint8_t *state[MAXB];   // current side
  int8_t *farSign[MAXB];
  uint8_t *hasDefW[MAXB];
  const void *vals[MAXB]; // current side
  int nBuf;
  int elem; // sizeof(T)
};

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

// err bits: 1 box too small (infinite direction), 4 pool capacity,
// 8 a freed brick still held a defined cell
__global__ void kMarkNeeded(GridDev g, const int *slotBrick, const int *slotList,
                            const int *nSlots, BufSet B, uint8_t *needed, int *err) {
  const int n = *nSlots;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int slot = slotList[i];
    bool core = false;
    for (int b = 0; b < B.nBuf; ++b) core |= B.hasDef[b][slot] != 0;
    if (!core) continue;
    int bx, by, bz;
    brickCoords(g, slotBrick[slot], bx, by, bz);
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
}

__global__ void kDilateBricks(GridDev g, int nBricks, const uint8_t *core,
                              uint8_t *needed, int *err) {
  for (int bi = blockIdx.x * blockDim.x + threadIdx.x; bi < nBricks;
       bi += gridDim.x * blockDim.x) {
    if (!core[bi]) continue;
    int bx, by, bz;
    brickCoords(g, bi, bx, by, bz);
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
}

template <class T>
__global__ void kFreeUnneeded(const int *slotList, const int *nSlots, int *brickMap,
                              int *slotBrick, const uint8_t *needed, BufSet B,
                              int *freeStack, int *freeCount, int *err) {
  const int n = *nSlots;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int slot = slotList[i];
    const int bi = slotBrick[slot];
    if (needed[bi]) continue;
    for (int b = 0; b < B.nBuf; ++b) {
      const uint8_t st = B.state[b][slot];
      int8_t s;
      if (st == ST_DENSE) {
        const T v = ((const T *)B.vals[b])[(size_t)slot * BV];
        if (isDef(v)) atomicOr(err, 8);
        s = v < 0 ? -1 : 1;
      } else {
        s = st == ST_UNEG ? -1 : 1;
      }
      B.farSign[b][bi] = s;
    }
    brickMap[bi] = -1;
    slotBrick[slot] = -1;
    freeStack[atomicAdd(freeCount, 1)] = slot;
  }
}

__global__ void kAllocNeeded(int nBricks, int *brickMap, int *slotBrick,
                             const uint8_t *needed, BufSet B, int *freeStack,
                             int *freeCount, int *err) {
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
    for (int b = 0; b < B.nBuf; ++b) {
      B.state[b][slot] = B.farSign[b][bi] < 0 ? ST_UNEG : ST_UPOS;
      B.hasDefW[b][slot] = 0;
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

__global__ void kFarSignFromRuns(GridDev g, int nBricks, const uint64_t *runKeys,
                                 const int8_t *runSign, int nRuns, int8_t *farSign) {
  for (int bi = blockIdx.x * blockDim.x + threadIdx.x; bi < nBricks;
       bi += gridDim.x * blockDim.x) {
    int bx, by, bz;
    brickCoords(g, bi, bx, by, bz);
    int x = g.org[0] + bx * BS + 4, y = g.org[1] + by * BS + 4, z = g.org[2] + bz * BS + 4;
    x = mapCoord(g, 0, x), y = mapCoord(g, 1, y), z = mapCoord(g, 2, z);
    farSign[bi] = runSignAt(runKeys, runSign, nRuns, cellKey(x, y, z)) < 0 ? -1 : 1;
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

template <class T>
__global__ void kFillFromRuns(GridDev g, const int *slotList, const int *nSlots,
                              const int *slotBrick, const uint64_t *runKeys,
                              const int8_t *runSign, int nRuns, T *vals) {
  const int n = *nSlots;
  for (int it = blockIdx.x; it < n; it += gridDim.x) {
    const int slot = slotList[it];
    int bx, by, bz;
    brickCoords(g, slotBrick[slot], bx, by, bz);
    for (int c = threadIdx.x; c < BV; c += blockDim.x) {
      int x = g.org[0] + bx * BS + (c & 7), y = g.org[1] + by * BS + ((c >> 3) & 7),
          z = g.org[2] + bz * BS + (c >> 6);
      x = mapCoord(g, 0, x), y = mapCoord(g, 1, y), z = mapCoord(g, 2, z);
      const int8_t s = runSignAt(runKeys, runSign, nRuns, cellKey(x, y, z));
      vals[(size_t)slot * BV + c] = s < 0 ? Lim<T>::lowest() : Lim<T>::max();
    }
  }
}

template <class T>
__global__ void kScatterPoints(GridDev g, int n, const int *idx, const double *v,
                               const int *brickMap, T *vals, int *err) {
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
    vals[(size_t)slot * BV + ((rz & 7) * 64 + (ry & 7) * 8 + (rx & 7))] = T(v[i]);
  }
}

// Set state / hasDef of every slot from its cells.
template <class T>
__global__ void kNormalize(GridDev g, const int *slotList, const int *nSlots,
                           const int *slotBrick, T *vals, uint8_t *state,
                           uint8_t *hasDef, unsigned long long *defCount) {
  const int n = *nSlots;
  for (int it = blockIdx.x; it < n; it += gridDim.x) {
    const int slot = slotList[it];
    int bx, by, bz;
    brickCoords(g, slotBrick[slot], bx, by, bz);
    bool anyDef = false, allPos = true, allNeg = true;
    for (int c = threadIdx.x; c < BV; c += blockDim.x) {
      const int x = g.org[0] + bx * BS + (c & 7), y = g.org[1] + by * BS + ((c >> 3) & 7),
                z = g.org[2] + bz * BS + (c >> 6);
      T v = vals[(size_t)slot * BV + c];
      if (!cellExists(g, x, y, z)) {
        vals[(size_t)slot * BV + c] = Lim<T>::max();
        continue;
      }
      if (isDef(v)) anyDef = true;
      else if (v < 0) allPos = false;
      else allNeg = false;
    }
    int nd = 0;
    for (int c = 0; c < BV; c += blockDim.x) {
      const int cc = c + threadIdx.x;
      const bool d = cc < BV && isDef(vals[(size_t)slot * BV + cc]);
      nd += __syncthreads_count(d);
    }
    if (threadIdx.x == 0 && nd) atomicAdd(defCount, (unsigned long long)nd);
    const int any = __syncthreads_or(anyDef);
    const int ap = __syncthreads_and(allPos);
    const int an = __syncthreads_and(allNeg);
    if (threadIdx.x == 0) {
      state[slot] = (!any && ap) ? ST_UPOS : ((!any && an) ? ST_UNEG : ST_DENSE);
      hasDef[slot] = any ? 1 : 0;
    }
  }
}

// Defined cells of a buffer as (HRLE key, value) pairs.
template <class T>
__global__ void kCompactDefined(GridDev g, const int *slotList, const int *nSlots,
                                const int *slotBrick, const T *vals,
                                const uint8_t *state, uint64_t *keys, double *out,
                                int *nOut, int room) {
  const int n = *nSlots;
  for (int it = blockIdx.x; it < n; it += gridDim.x) {
    const int slot = slotList[it];
    if (state[slot] != ST_DENSE) continue;
    int bx, by, bz;
    brickCoords(g, slotBrick[slot], bx, by, bz);
    for (int k = 0; k < BV / 256; ++k) {
      const int c = threadIdx.x + k * 256;
      const int x = g.org[0] + bx * BS + (c & 7), y = g.org[1] + by * BS + ((c >> 3) & 7),
                z = g.org[2] + bz * BS + (c >> 6);
      const T v = vals[(size_t)slot * BV + c];
      const bool d = isDef(v) && cellExists(g, x, y, z);
      const unsigned mask = __ballot_sync(0xffffffffu, d);
      const int lane = threadIdx.x & 31;
      int off = 0;
      if (lane == 0 && mask) off = atomicAdd(nOut, __popc(mask));
      off = __shfl_sync(0xffffffffu, off, 0);
      const int p = off + __popc(mask & ((1u << lane) - 1));
      if (d && p < room) {
        keys[p] = cellKey(x, y, z);
        out[p] = (double)v;
      }
    }
  }
}

template <class T>
__global__ void kQueryValues(GridDev g, MapView m, Buf<T> b, int n, const int *idx,
                             double *out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const T v = cellValueRaw<T>(g, m, b, idx[3 * i], idx[3 * i + 1], idx[3 * i + 2]);
    out[i] = isDef(v) ? (double)v : (v < 0 ? -DBL_MAX : DBL_MAX);
  }
}

template <class T>
__global__ void kCountDefined(const int *slotList, const int *nSlots, const T *vals,
                              const uint8_t *state, unsigned long long *cnt) {
  const int n = *nSlots;
  for (int it = blockIdx.x; it < n; it += gridDim.x) {
    const int slot = slotList[it];
    if (state[slot] != ST_DENSE) continue;
    int nd = 0;
    for (int c = 0; c < BV; c += blockDim.x)
      nd += __syncthreads_count(isDef(vals[(size_t)slot * BV + c + threadIdx.x]));
    if (threadIdx.x == 0 && nd) atomicAdd(cnt, (unsigned long long)nd);
  }
}

// Copy the listed slots of one buffer into another (RK initial copies).
template <class T>
__global__ void kCopySlots(const int *slotList, const int *nSlots, const T *sv,
                           const uint8_t *ss, const uint8_t *sh, T *dv, uint8_t *ds,
                           uint8_t *dh) {
  const int n = *nSlots;
  for (int it = blockIdx.x; it < n; it += gridDim.x) {
    const int slot = slotList[it];
    const uint8_t st = ss[slot];
    if (threadIdx.x == 0) {
      ds[slot] = st;
      dh[slot] = sh[slot];
    }
    if (st == ST_DENSE)
      for (int c = threadIdx.x; c < BV; c += blockDim.x)
        dv[(size_t)slot * BV + c] = sv[(size_t)slot * BV + c];
  }
}

} // namespace vlsg
