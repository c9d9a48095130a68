// vlsg_exchange.cuh -- the exchange format of a level set built on the
// device: its defined points in HRLE order (z, then y, then x; the order
// viennahrle's iterators visit them, lsDomain.hpp) and its undefined runs
// with their signs.
//
// Points: the allocated bricks are listed in brick order (bz, by, bx).  A
// "segment" is one x-row of one brick (8 cells: brick i, plane lz, row ly);
// in HRLE order the segments come as (bz, lz, by, ly, bx), so segment
// (i, lz, ly) of a brick in slab [s0, s1) (bricks with its bz) and brick row
// [r0, r1) (bricks with its bz, by) has the rank
//   64 s0 + 8 lz (s1 - s0) + 8 (r0 - s0) + ly (r1 - r0) + (i - r0).
// An exclusive scan of the segments' point counts in that order gives every
// segment its output offset -- no sort.
//
// Runs: over the box [min - 1, max + 1] of the points, in HRLE order: one run
// before the box, per plane one run before its rows, per row a head run (or
// one run for a row without points) and a run after every point that is not
// followed by its +x neighbour, per plane one run after its rows, one run
// after the box.  Each takes the sign of the level set at a cell inside it;
// runs that repeat the previous sign with no defined point between are
// dropped.  With row r = zi * NY + yi and G gap runs before a given one,
//   head(r) = 2 + 2 zi + r + GB(r),   gap run = 3 + 2 zi + r + G,
// where GB(r) counts the gap runs of the rows before r.
#pragma once

#include "vlsg_common.cuh"
#include "vlsg_frontier.cuh"
#include "vlsg_maint.cuh"
#include "vlsg_scan.cuh"

namespace vlsg {
namespace { // internal linkage: every compilation unit has its own copy

constexpr int XNI = -((1 << 20) - 2); // start index of runs that begin at -infinity

__global__ void kAllocFlags(const int *brickMap, int nBricks, uint32_t *f) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nBricks; b += gridDim.x * blockDim.x)
    f[b] = brickMap[b] >= 0 ? 1u : 0u;
}

__global__ void kOrderedBricks(const int *brickMap, int nBricks, const uint32_t *pos, int *ob) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nBricks; b += gridDim.x * blockDim.x)
    if (brickMap[b] >= 0) ob[pos[b]] = b;
}

__device__ inline int lowerBound(const int *a, int n, int key) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (a[mid] < key) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// Brick row [r0, r1) and slab [s0, s1) of every ordered brick.
__global__ void kBrickBounds(GridDev g, const int *ob, int nAlloc, int4 *bounds) {
  const int rowLen = g.nb[0], slabLen = g.nb[0] * g.nb[1];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nAlloc; i += gridDim.x * blockDim.x) {
    const int bi = ob[i];
    const int row = bi / rowLen, slab = bi / slabLen;
    int4 b;
    b.x = lowerBound(ob, nAlloc, row * rowLen);
    b.y = lowerBound(ob, nAlloc, (row + 1) * rowLen);
    b.z = lowerBound(ob, nAlloc, slab * slabLen);
    b.w = lowerBound(ob, nAlloc, (slab + 1) * slabLen);
    bounds[i] = b;
  }
}

__device__ inline uint32_t segmentRank(const int4 &b, int i, int lz, int ly) {
  return 64u * b.z + 8u * lz * (b.w - b.z) + 8u * (b.x - b.z) + (uint32_t)ly * (b.y - b.x) +
         (i - b.x);
}

// Byte of the defined mask for segment (lz, ly) of a slot.
__device__ inline unsigned segByte(const uint64_t *def, int slot, int lz, int ly) {
  return (unsigned)((def[(size_t)slot * 8 + lz] >> (8 * ly)) & 0xffull);
}

// Point count of every segment (at its rank) and the bounding box of the
// points (atomic min / max of x, y, z into box[0..5]).
__global__ void kSegCounts(GridDev g, const int *ob, int nAlloc, const int *brickMap,
                           const int4 *bounds, const uint64_t *def, uint32_t *C, int *box) {
  const size_t nSeg = (size_t)nAlloc * 64;
  int mn[3] = {INT_MAX, INT_MAX, INT_MAX}, mx[3] = {INT_MIN, INT_MIN, INT_MIN};
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < nSeg;
       e += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(e >> 6), lz = (int)(e >> 3) & 7, ly = (int)e & 7;
    const int bi = ob[i];
    const unsigned byte = segByte(def, brickMap[bi], lz, ly);
    C[segmentRank(bounds[i], i, lz, ly)] = __popc(byte);
    if (byte) {
      int bx, by, bz;
      brickCoords(g, bi, bx, by, bz);
      const int x0 = g.org[0] + bx * BS, y = g.org[1] + by * BS + ly, z = g.org[2] + bz * BS + lz;
      mn[0] = min(mn[0], x0 + __ffs(byte) - 1);
      mx[0] = max(mx[0], x0 + 31 - __clz(byte));
      mn[1] = min(mn[1], y), mx[1] = max(mx[1], y);
      mn[2] = min(mn[2], z), mx[2] = max(mx[2], z);
    }
  }
  for (int d = 0; d < 3; ++d) {
    for (int o = 16; o > 0; o >>= 1) {
      mn[d] = min(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], o));
      mx[d] = max(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], o));
    }
  }
  if ((threadIdx.x & 31) == 0 && mn[0] != INT_MAX) {
    for (int d = 0; d < 3; ++d) {
      atomicMin(&box[d], mn[d]);
      atomicMax(&box[3 + d], mx[d]);
    }
  }
}

// Box of the runs: [min - 1, max + 1] of the points (or the origin).
struct RunBox {
  int lo[3], hi[3];
  int ny, nz;
  __device__ int rowOf(int y, int z) const { return (z - lo[2]) * ny + (y - lo[1]); }
};

// Points of every segment at their offsets, in x order; gap runs per segment
// (points not followed by their +x neighbour) at their rank, and per row the
// point and gap-run counts.
template <class T>
__global__ void kSegScatter(GridDev g, const int *ob, int nAlloc, const int *brickMap,
                            const int *nbr, const int4 *bounds, const uint64_t *def,
                            const T *vals, const uint32_t *P, RunBox rb, int32_t *idxOut,
                            double *valOut, uint32_t *GC, uint32_t *rowCount, uint32_t *rowGaps,
                            const float *lo) {
  const size_t nSeg = (size_t)nAlloc * 64;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < nSeg;
       e += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(e >> 6), lz = (int)(e >> 3) & 7, ly = (int)e & 7;
    const int bi = ob[i];
    const int slot = brickMap[bi];
    const unsigned byte = segByte(def, slot, lz, ly);
    const uint32_t rank = segmentRank(bounds[i], i, lz, ly);
    if (!byte) {
      GC[rank] = 0;
      continue;
    }
    int bx, by, bz;
    brickCoords(g, bi, bx, by, bz);
    const int x0 = g.org[0] + bx * BS, y = g.org[1] + by * BS + ly, z = g.org[2] + bz * BS + lz;
    // is the +x neighbour brick's first cell of this row defined?
    bool nextFirst = false;
    if (bx + 1 < g.nb[0]) {
      const int s = nbr[(size_t)slot * 27 + NB_XP];
      if (s >= 0) nextFirst = segByte(def, s, lz, ly) & 1u;
    }
    uint32_t pos = P[rank];
    unsigned gaps = 0;
    for (unsigned m = byte; m; m &= m - 1) {
      const int lx = __ffs(m) - 1;
      idxOut[3 * (size_t)pos + 0] = x0 + lx;
      idxOut[3 * (size_t)pos + 1] = y;
      idxOut[3 * (size_t)pos + 2] = z;
      const size_t q = (size_t)slot * BV + lz * 64 + ly * 8 + lx;
      // with a compensation term the value is hi + lo
      valOut[pos] = lo ? withLo((double)vals[q], lo[q]) : (double)vals[q];
      ++pos;
      const bool adjacent = lx < 7 ? ((byte >> (lx + 1)) & 1u) : nextFirst;
      gaps += adjacent ? 0u : 1u;
    }
    GC[rank] = gaps;
    const int r = rb.rowOf(y, z);
    atomicAdd(&rowCount[r], (uint32_t)__popc(byte));
    atomicAdd(&rowGaps[r], gaps);
  }
}

__device__ inline int floorDiv2(int a) { return a >= 0 ? a / 2 : -((-a + 1) / 2); }

template <class T> struct RunSink {
  int32_t *start; // 3 per run
  int8_t *sign;
  uint32_t *pb;   // defined points before the run (for the merge of equal runs)
  GridDev g;
  MapView m;
  Buf<T> b;
  __device__ void put(uint32_t k, int x, int y, int z, int px, int py, int pz, uint32_t before) const {
    start[3 * (size_t)k + 0] = x;
    start[3 * (size_t)k + 1] = y;
    start[3 * (size_t)k + 2] = z;
    const T v = cellValueRaw<T>(g, m, b, px, py, pz);
    sign[k] = v < 0 ? -1 : 1;
    pb[k] = before;
  }
};

// Row, plane and box runs (one thread per row of the run box).
template <class T>
__global__ void kRunsRows(RunBox rb, const uint32_t *rowCount, const uint32_t *rowGaps,
                          const uint32_t *PB, const uint32_t *GB, const int32_t *idxOut,
                          uint32_t nPoints, uint32_t nRuns, RunSink<T> sink) {
  const int rows = rb.ny * rb.nz;
  const int cx = floorDiv2(rb.lo[0] + rb.hi[0]), cy = floorDiv2(rb.lo[1] + rb.hi[1]);
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x) {
    const int zi = r / rb.ny, yi = r % rb.ny;
    const int z = rb.lo[2] + zi, y = rb.lo[1] + yi;
    const uint32_t head = 2u + 2u * zi + (uint32_t)r + GB[r];
    if (rowCount[r] == 0) {
      sink.put(head, XNI, y, z, rb.lo[0], y, z, PB[r]);
    } else {
      const int fx = idxOut[3 * (size_t)PB[r]];
      sink.put(head, XNI, y, z, fx - 1, y, z, PB[r]);
    }
    if (yi == 0) sink.put(head - 1, XNI, XNI, z, cx, rb.lo[1] - 1, z, PB[r]);
    if (yi == rb.ny - 1)
      sink.put(head + 1 + rowGaps[r], XNI, rb.hi[1] + 1, z, cx, rb.hi[1] + 1, z,
               PB[r] + rowCount[r]);
    if (r == 0) sink.put(0, XNI, XNI, XNI, cx, cy, rb.lo[2] - 1, 0);
    if (r == rows - 1) sink.put(nRuns - 1, XNI, XNI, rb.hi[2] + 1, cx, cy, rb.hi[2] + 1, nPoints);
  }
}

// Gap runs (one thread per segment): after every point not followed by its
// +x neighbour.
template <class T>
__global__ void kRunsGaps(GridDev g, const int *ob, int nAlloc, const int *brickMap,
                          const int *nbr, const int4 *bounds, const uint64_t *def,
                          const uint32_t *P, const uint32_t *GE, RunBox rb, RunSink<T> sink) {
  const size_t nSeg = (size_t)nAlloc * 64;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < nSeg;
       e += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(e >> 6), lz = (int)(e >> 3) & 7, ly = (int)e & 7;
    const int bi = ob[i];
    const int slot = brickMap[bi];
    const unsigned byte = segByte(def, slot, lz, ly);
    if (!byte) continue;
    const uint32_t rank = segmentRank(bounds[i], i, lz, ly);
    int bx, by, bz;
    brickCoords(g, bi, bx, by, bz);
    const int x0 = g.org[0] + bx * BS, y = g.org[1] + by * BS + ly, z = g.org[2] + bz * BS + lz;
    bool nextFirst = false;
    if (bx + 1 < g.nb[0]) {
      const int s = nbr[(size_t)slot * 27 + NB_XP];
      if (s >= 0) nextFirst = segByte(def, s, lz, ly) & 1u;
    }
    const int r = rb.rowOf(y, z);
    const int zi = z - rb.lo[2];
    uint32_t k = 3u + 2u * zi + (uint32_t)r + GE[rank];
    uint32_t p = P[rank];
    for (unsigned m = byte; m; m &= m - 1) {
      const int lx = __ffs(m) - 1;
      ++p;
      const bool adjacent = lx < 7 ? ((byte >> (lx + 1)) & 1u) : nextFirst;
      if (!adjacent) {
        sink.put(k, x0 + lx + 1, y, z, x0 + lx + 1, y, z, p);
        ++k;
      }
    }
  }
}

// Runs kept by the merge: the first, and every one whose sign or number of
// points before differs from its predecessor's.
__global__ void kRunKeep(const int8_t *sign, const uint32_t *pb, uint32_t n, uint32_t *keep) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    keep[i] = (i == 0 || sign[i] != sign[i - 1] || pb[i] != pb[i - 1]) ? 1u : 0u;
}

__global__ void kRunCompact(const int32_t *start, const int8_t *sign, const uint32_t *keep,
                            const uint32_t *pos, uint32_t n, int32_t *outStart, int8_t *outSign) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (!keep[i]) continue;
    const uint32_t o = pos[i];
    outStart[3 * (size_t)o + 0] = start[3 * (size_t)i + 0];
    outStart[3 * (size_t)o + 1] = start[3 * (size_t)i + 1];
    outStart[3 * (size_t)o + 2] = start[3 * (size_t)i + 2];
    outSign[o] = sign[i];
  }
}

} // namespace
} // namespace vlsg
