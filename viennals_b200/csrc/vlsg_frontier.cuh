// vlsg_frontier.cuh -- band passes that evaluate only the cells that can
// change.
//
// Every level-set buffer keeps, per allocated 8^3 brick, the values of all
// its cells (updated in place) and a 512-bit mask of its defined cells (one
// 64-bit word per z-plane, bit y*8+x).  A pass takes one warp per brick,
// finds the brick's candidate cells by bit dilation of the masks (neighbour
// bricks' face planes through the 27-neighbour table), evaluates the
// reference's rule on the candidates only and appends every (cell, new value)
// that changes to its warp's own segment of a change log (no atomics: a warp
// handles at most ceil(slots / warps) bricks of 512 cells); kApplyChanges
// streams the log back afterwards, so every rule reads old values only --
// the reference maps the whole old level set to a new one (Jacobi order).
// The new defined masks go to a second mask array.
// Candidates per pass:
//   Expand (lsExpand.hpp:104-157): undefined cells next to a defined one.  A
//     defined cell keeps its value when |v| <= width/2, which the engine
//     tracks per buffer; otherwise the defined cells are candidates too.
//   Prune (lsPrune.hpp:118-180): the defined cells (undefined ones keep their
//     sentinel).
//   rebuildLS (lsAdvect.hpp:299-415): defined cells and their neighbours (an
//     undefined cell with no defined neighbour keeps its sentinel).
//   updateLevelSet + rebuildLS: after Reduce(1) (lsReduce.hpp:285-296) the
//     defined cells are the active ones; candidates are the active cells and
//     their neighbours, and every other defined cell becomes undefined with
//     its sign.
// Bricks next to a boundary that remaps cells (reflective, periodic with a
// length that is not a multiple of 8, the mirrored side of POS/NEG_INFINITE)
// are "complex": all their existing cells are candidates and their
// neighbours are read through the boundary mapping.
#pragma once

#include "vlsg_common.cuh"
#include "vlsg_passes.cuh"

namespace vlsg {
namespace { // internal linkage: every compilation unit has its own copy

constexpr int FRONTIER_THREADS = 256;
// Resident blocks per SM the passes are compiled for (40 registers per
// thread): the passes are bound by latency and issue, so occupancy pays more
// than the few spilled registers cost.
#ifndef VLSG_PASS_MIN_BLOCKS
#define VLSG_PASS_MIN_BLOCKS 6
#endif
constexpr uint64_t XLO = 0x0101010101010101ull; // cells with x = 0
constexpr uint64_t XHI = 0x8080808080808080ull; // cells with x = 7
// 27-neighbour table entries of the six faces (index (dz+1)*9+(dy+1)*3+dx+1)
constexpr int NB_XM = 12, NB_XP = 14, NB_YM = 10, NB_YP = 16, NB_ZM = 4, NB_ZP = 22;
constexpr uint8_t CF_STAR = 1; // a star neighbour of a cell is remapped
constexpr uint8_t CF_NEAR = 2; // a cell within 8 cells is remapped

// Brick topology shared by the passes.
struct Topo {
  GridDev g;
  const int *brickMap, *slotBrick, *slotList, *nSlots;
  const int *nbr;       // 27 entries per slot: slot, or -1-brick
  const uint8_t *cflag; // CF_* per slot
  int *err;
};

// Point data carried by the cells of the top level set (null arrays: none):
// the source id of the data a defined cell carries (the index of a point at
// the start of the advection, -1: none) and the saved advection velocity and
// dissipation (lsAdvect.hpp:780-796).  In a change log the same arrays hold
// the data of each logged cell.
template <class T> struct Payload {
  int32_t *src;
  T *vel, *diss;
};

template <class T> struct LsView {
  T *vals;               // slots x 512 cells, in place
  const uint64_t *def;   // current masks, slots x 8 words
  uint64_t *defNext;     // masks after the pass
  const int8_t *farSign; // per brick of the map box
  Payload<T> pd;         // point data per cell, or null arrays
};

// Change log: segment w (of `per` entries) belongs to warp w of the pass.
template <class T> struct ChangeLog {
  uint32_t *cell; // slot << 9 | cell
  T *val;
  int *count;     // entries per segment
  size_t per;
  Payload<T> pd;  // point data per entry (with a view that carries it)
};

// Point data of the value a rule produced: src -1 keeps the centre's, 0..5
// takes star neighbour src's (cell loc of slot ref), -2 none.
template <class T>
__device__ inline void payloadOf(const Payload<T> &pd, size_t centre, int src, int ref, int loc,
                                 int32_t &s, T &v, T &d) {
  if (src == -1) {
    s = pd.src[centre], v = pd.vel[centre], d = pd.diss[centre];
  } else if (src >= 0 && ref >= 0) {
    const size_t q = (size_t)ref * BV + loc;
    s = pd.src[q], v = pd.vel[q], d = pd.diss[q];
  } else {
    s = -1, v = T(0), d = T(0);
  }
}

template <class T> __device__ inline T sentinel(bool neg) {
  return neg ? Lim<T>::lowest() : Lim<T>::max();
}

// Slot (or -1-brick) and cell index of global cell (x,y,z) through the
// boundary mapping; cells outside the map box take the nearest box cell.
__device__ inline int locateCell(const GridDev &g, const int *brickMap, int x, int y, int z,
                                 int &local) {
  x = mapCoord(g, 0, x), y = mapCoord(g, 1, y), z = mapCoord(g, 2, z);
  int rx = x - g.org[0], ry = y - g.org[1], rz = z - g.org[2];
  const int ex = g.nb[0] * BS - 1, ey = g.nb[1] * BS - 1, ez = g.nb[2] * BS - 1;
  rx = rx < 0 ? 0 : (rx > ex ? ex : rx);
  ry = ry < 0 ? 0 : (ry > ey ? ey : ry);
  rz = rz < 0 ? 0 : (rz > ez ? ez : rz);
  const int bi = brickIndex(g, rx >> 3, ry >> 3, rz >> 3);
  local = (rz & 7) * 64 + (ry & 7) * 8 + (rx & 7);
  const int slot = brickMap[bi];
  return slot >= 0 ? slot : -1 - bi;
}

// Face neighbours of a slot in the 27-table order -x,+x,-y,+y,-z,+z.
__device__ inline int faceEntry(int f) {
  return f == 0 ? NB_XM : f == 1 ? NB_XP : f == 2 ? NB_YM : f == 3 ? NB_YP : f == 4 ? NB_ZM : NB_ZP;
}

// Per-warp shared scratch of the brick in hand.
struct WarpScratch {
  unsigned long long flip[8]; // cells whose definedness flips
  int nb[6];                  // face neighbours -x,+x,-y,+y,-z,+z (slot or -1-brick)
  int pad[2];
  unsigned long long aux[8];  // a second mask of the brick (kUpdateRebuild: active cells)
  uint16_t list[BV];          // the brick's cells to evaluate, ascending
};

// Start of a brick: face neighbours to shared memory, flips cleared.
__device__ inline void beginBrick(const Topo &t, WarpScratch &ws, int slot, int lane) {
  if (lane < 6) ws.nb[lane] = t.nbr[(size_t)slot * 27 + faceEntry(lane)];
  if (lane < 8) ws.flip[lane] = 0ull;
  __syncwarp();
}

// Publish the brick's new defined mask (old ^ flips) and, when `visit` is
// given, mark the bricks the next pass of this buffer must visit: this one if
// it holds a defined cell, and each face neighbour with a defined cell of this
// brick on the shared face (only those can have candidate cells).
__device__ inline void finishBrick(WarpScratch &ws, uint64_t *defNext, int slot, int lane,
                                   uint64_t own, uint8_t *visit) {
  __syncwarp();
  const uint64_t nw = lane < 8 ? own ^ ws.flip[lane] : 0ull;
  if (lane < 8) defNext[(size_t)slot * 8 + lane] = nw;
  if (visit) {
    const unsigned self = __ballot_sync(0xffffffffu, nw != 0ull);
    const unsigned xm = __ballot_sync(0xffffffffu, (nw & XLO) != 0ull);
    const unsigned xp = __ballot_sync(0xffffffffu, (nw & XHI) != 0ull);
    const unsigned ym = __ballot_sync(0xffffffffu, (nw & 0xffull) != 0ull);
    const unsigned yp = __ballot_sync(0xffffffffu, (nw >> 56) != 0ull);
    if (lane == 0 && self) {
      visit[slot] = 1;
      if (xm && ws.nb[0] >= 0) visit[ws.nb[0]] = 1;
      if (xp && ws.nb[1] >= 0) visit[ws.nb[1]] = 1;
      if (ym && ws.nb[2] >= 0) visit[ws.nb[2]] = 1;
      if (yp && ws.nb[3] >= 0) visit[ws.nb[3]] = 1;
      if ((self & 1u) && ws.nb[4] >= 0) visit[ws.nb[4]] = 1;
      if ((self & 0x80u) && ws.nb[5] >= 0) visit[ws.nb[5]] = 1;
    }
  }
  __syncwarp();
}

__device__ inline void brickOrigin(const Topo &t, int slot, int &x0, int &y0, int &z0) {
  int bx, by, bz;
  brickCoords(t.g, t.slotBrick[slot], bx, by, bz);
  x0 = t.g.org[0] + bx * BS, y0 = t.g.org[1] + by * BS, z0 = t.g.org[2] + bz * BS;
}

// Star neighbour j (order +x,+y,+z,-x,-y,-z) of local cell c as (slot or
// -1-brick, cell): through the face neighbours, or, for a brick next to a
// boundary that remaps cells, through the brick map and the mapping.
__device__ inline int starRef(const Topo &t, const int *nb, int slot, bool complex, int x0,
                              int y0, int z0, int c, int j, int &loc) {
  const int x = c & 7, y = (c >> 3) & 7, z = c >> 6;
  if (complex) {
    const int dx = j == 0 ? 1 : j == 3 ? -1 : 0, dy = j == 1 ? 1 : j == 4 ? -1 : 0,
              dz = j == 2 ? 1 : j == 5 ? -1 : 0;
    return locateCell(t.g, t.brickMap, x0 + x + dx, y0 + y + dy, z0 + z + dz, loc);
  }
  switch (j) {
  case 0: loc = x < 7 ? c + 1 : c - 7; return x < 7 ? slot : nb[1];
  case 1: loc = y < 7 ? c + 8 : c - 56; return y < 7 ? slot : nb[3];
  case 2: loc = z < 7 ? c + 64 : c - 448; return z < 7 ? slot : nb[5];
  case 3: loc = x > 0 ? c - 1 : c + 7; return x > 0 ? slot : nb[0];
  case 4: loc = y > 0 ? c - 8 : c + 56; return y > 0 ? slot : nb[2];
  default: loc = z > 0 ? c - 64 : c + 448; return z > 0 ? slot : nb[4];
  }
}

template <class T>
__device__ inline T refValue(const T *vals, const int8_t *farSign, int ref, int loc) {
  return ref >= 0 ? vals[(size_t)ref * BV + loc] : sentinel<T>(farSign[-1 - ref] < 0);
}

// Mask of the cells of plane z that exist in the grid.
__device__ inline uint64_t existPlane(const GridDev &g, int x0, int y0, int z0, int z) {
  uint64_t m = 0;
  for (int y = 0; y < 8; ++y)
    for (int x = 0; x < 8; ++x)
      if (cellExists(g, x0 + x, y0 + y, z0 + z)) m |= 1ull << (y * 8 + x);
  return m;
}

// Star dilation of the brick's mask, plane of lane z (lanes 0..7; the other
// lanes return 0).  Every lane of the warp must call it.  Sets err bit 64
// when a set cell lies on a face whose neighbour brick is not allocated
// (its cells could change but are not in the pool).
__device__ inline uint64_t dilatedMask(const Topo &t, const uint64_t *mask, int slot,
                                       const int *nb, int lane) {
  const int z = lane & 7;
  const uint64_t w = lane < 8 ? mask[(size_t)slot * 8 + z] : 0ull;
  uint64_t below = __shfl_sync(0xffffffffu, w, (z + 7) & 7);
  uint64_t above = __shfl_sync(0xffffffffu, w, (z + 1) & 7);
  if (lane >= 8) return 0ull;
  if (z == 0) below = nb[4] >= 0 ? mask[(size_t)nb[4] * 8 + 7] : 0ull;
  if (z == 7) above = nb[5] >= 0 ? mask[(size_t)nb[5] * 8 + 0] : 0ull;
  const uint64_t nxm = nb[0] >= 0 ? mask[(size_t)nb[0] * 8 + z] : 0ull;
  const uint64_t nxp = nb[1] >= 0 ? mask[(size_t)nb[1] * 8 + z] : 0ull;
  const uint64_t nym = nb[2] >= 0 ? mask[(size_t)nb[2] * 8 + z] : 0ull;
  const uint64_t nyp = nb[3] >= 0 ? mask[(size_t)nb[3] * 8 + z] : 0ull;
  const bool open = ((w & XLO) && nb[0] < 0) || ((w & XHI) && nb[1] < 0) ||
                    ((w & 0xffull) && nb[2] < 0) || ((w >> 56) && nb[3] < 0) ||
                    (z == 0 && w && nb[4] < 0) || (z == 7 && w && nb[5] < 0);
  if (open) atomicOr(t.err, 64);
  return w | ((w << 1) & ~XLO) | ((w >> 1) & ~XHI) | ((nxm & XHI) >> 7) | ((nxp & XLO) << 7) |
         (w << 8) | (w >> 8) | (nym >> 56) | (nyp << 56) | below | above;
}

// List the set cells of a brick mask (lane z holds plane z, z < 8) into
// `list` in ascending order: lane l < 16 walks the 32-bit half l & 1 of plane
// l >> 1.  Returns the number of cells (every lane).  Every lane of the warp
// must call it.
__device__ inline int listCells(uint64_t plane, uint16_t *list) {
  const int lane = threadIdx.x & 31;
  const uint64_t pw = __shfl_sync(0xffffffffu, plane, lane >> 2);
  unsigned w = (unsigned)(pw >> (16 * (lane & 3))) & 0xffffu;
  const int cnt = __popc(w);
  int x = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += t;
  }
  int off = x - cnt;
  const int total = __shfl_sync(0xffffffffu, x, 31);
  const int base = (lane >> 2) * 64 + (lane & 3) * 16;
  while (w) {
    list[off++] = (uint16_t)(base + __ffs(w) - 1);
    w &= w - 1;
  }
  __syncwarp();
  return total;
}

__device__ inline void markCell(unsigned long long *words, int c) {
  // the 32-bit half of the plane word that holds the cell (little endian)
  atomicOr(reinterpret_cast<unsigned *>(words) + (c >> 5), 1u << (c & 31));
}

// Append the lanes with `has` to the warp's log segment (warp-uniform call),
// with the point data (ps, pv, pdi) when the log carries it.
template <class T>
__device__ inline void logChange(const ChangeLog<T> &lg, size_t base, int &count, bool has,
                                 uint32_t cell, T val, int32_t ps = -1, T pv = T(0),
                                 T pdi = T(0)) {
  const unsigned m = __ballot_sync(0xffffffffu, has);
  if (has) {
    const size_t p = base + count + __popc(m & ((1u << (threadIdx.x & 31)) - 1));
    lg.cell[p] = cell;
    lg.val[p] = val;
    if (lg.pd.src) lg.pd.src[p] = ps, lg.pd.vel[p] = pv, lg.pd.diss[p] = pdi;
  }
  count += __popc(m);
}

enum : int { FP_EXPAND = 0, FP_PRUNE = 1, FP_ALL = 2 };

// One brick of a star pass of a rule (one warp): candidates, evaluation,
// change log, new masks and visit flags.  MODE picks the candidates:
// FP_EXPAND undefined cells next to a defined one, FP_PRUNE the defined
// cells, FP_ALL the defined cells and their neighbours.
template <class T, int MODE, class Rule>
__device__ inline void frontierBrick(const Topo &t, const LsView<T> &v, const Rule &rule,
                                     const ChangeLog<T> &lg, WarpScratch &ws, int slot,
                                     bool complex, uint64_t own, size_t logBase, int &logged,
                                     uint8_t *visitOut, bool &zeroHit) {
  const int lane = threadIdx.x & 31;
  beginBrick(t, ws, slot, lane);
  int x0 = 0, y0 = 0, z0 = 0;
  if (complex) brickOrigin(t, slot, x0, y0, z0);
  uint64_t cand;
  if (MODE == FP_PRUNE) {
    cand = own;
  } else if (complex) {
    const uint64_t ex = lane < 8 ? existPlane(t.g, x0, y0, z0, lane) : 0ull;
    cand = MODE == FP_EXPAND ? ex & ~own : ex;
  } else {
    const uint64_t dil = dilatedMask(t, v.def, slot, ws.nb, lane);
    cand = MODE == FP_EXPAND ? dil & ~own : dil;
  }
  const int total = __any_sync(0xffffffffu, cand != 0ull) ? listCells(cand, ws.list) : 0;
  for (int base = 0; base < total; base += 32) {
    const int k = base + lane;
    bool changed = false;
    T out = T(0);
    int c = 0;
    int32_t ps = -1;
    T pv = T(0), pdi = T(0);
    if (k < total) {
      c = ws.list[k];
      const T center = v.vals[(size_t)slot * BV + c];
      if (MODE == FP_PRUNE && center == T(0)) zeroHit = true;
      T nb[6];
#pragma unroll
      for (int j = 0; j < 6; ++j) {
        int loc;
        const int ref = starRef(t, ws.nb, slot, complex, x0, y0, z0, c, j, loc);
        nb[j] = refValue<T>(v.vals, v.farSign, ref, loc);
      }
      int src = -1;
      out = rule(center, nb, src);
      changed = out != center || signbit(out) != signbit(center);
      if (changed && isDef(out) != isDef(center)) markCell(ws.flip, c);
      // with point data a value taken from a neighbour is logged even when
      // it equals the old one: its data changes
      if (lg.pd.src && isDef(out) && src >= 0) changed = true;
      if (changed && lg.pd.src && isDef(out)) {
        int loc = 0, ref = -1;
        if (src >= 0) ref = starRef(t, ws.nb, slot, complex, x0, y0, z0, c, src, loc);
        payloadOf<T>(v.pd, (size_t)slot * BV + c, src, ref, loc, ps, pv, pdi);
      }
    }
    logChange<T>(lg, logBase, logged, changed, ((uint32_t)slot << 9) | (uint32_t)c, out, ps, pv,
                 pdi);
  }
  finishBrick(ws, v.defNext, slot, lane, own, visitOut);
}

template <class T, int MODE, class Rule>
__global__ void __launch_bounds__(FRONTIER_THREADS, VLSG_PASS_MIN_BLOCKS)
    kFrontierPass(Topo t, LsView<T> v, Rule rule, ChangeLog<T> lg, const uint8_t *visitIn,
                  uint8_t *visitOut, int *zeros, int zeroMode, int poolSlots) {
  __shared__ WarpScratch sm[FRONTIER_THREADS / 32];
  WarpScratch &ws = sm[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nWarps = (gridDim.x * blockDim.x) >> 5;
  const int n = *t.nSlots;
  const size_t logBase = (size_t)warp * lg.per;
  int logged = 0;
  // zeroMode 1: record a defined candidate +-0 in *zeros; zeroMode 2: when
  // *zeros is 0 the pass is known to change nothing (the second Prune of a
  // pair): copy the masks and the visit flags of the whole pool (free slots
  // included, whose contents no one reads), log nothing
  if (MODE == FP_PRUNE && zeroMode == 2 && *zeros == 0) {
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t nThreads = (size_t)gridDim.x * blockDim.x;
    const uint4 *src = reinterpret_cast<const uint4 *>(v.def); // 4 x 16 bytes per slot
    uint4 *dst = reinterpret_cast<uint4 *>(v.defNext);
    for (size_t i = tid; i < (size_t)poolSlots * 4; i += nThreads) dst[i] = src[i];
    if (visitOut)
      for (size_t i = tid; i < (size_t)poolSlots; i += nThreads)
        visitOut[i] = visitIn ? visitIn[i] : 1;
    if (lane == 0) lg.count[warp] = 0;
    return;
  }
  bool zeroHit = false;
  for (int w = warp; w < n; w += nWarps) {
    const int slot = t.slotList[w];
    const bool complex = (t.cflag[slot] & CF_STAR) != 0;
    // a brick the previous pass of this buffer did not mark has no defined
    // cell and no defined face neighbour cell: nothing to evaluate
    if (visitIn && !complex && !visitIn[slot]) {
      if (lane < 8) v.defNext[(size_t)slot * 8 + lane] = 0ull;
      continue;
    }
    const uint64_t own = lane < 8 ? v.def[(size_t)slot * 8 + lane] : 0ull;
    if (MODE == FP_PRUNE && !complex && !__any_sync(0xffffffffu, own != 0ull)) {
      if (lane < 8) v.defNext[(size_t)slot * 8 + lane] = 0ull;
      continue;
    }
    frontierBrick<T, MODE, Rule>(t, v, rule, lg, ws, slot, complex, own, logBase, logged, visitOut,
                                 zeroHit);
  }
  if (lane == 0) lg.count[warp] = logged;
  if (MODE == FP_PRUNE && zeroMode == 1 && __any_sync(0xffffffffu, zeroHit) && lane == 0)
    atomicOr(zeros, 1);
}

// Write a change log back: warp w copies segment w.
// `lo` (FP32 buffers that carry a compensation term, else null): a cell a
// pass changed holds a value computed from the stored values alone, so its
// compensation term becomes 0.
template <class T>
__global__ void __launch_bounds__(FRONTIER_THREADS)
    kApplyChanges(T *vals, ChangeLog<T> lg, int segments, float *lo, Payload<T> pd) {
  // block b takes segments b, b + gridDim.x, ...; its 256 threads stride the
  // entries, four loads in flight per thread
  for (int w = blockIdx.x; w < segments; w += gridDim.x) {
    const int n = lg.count[w];
    const size_t base = (size_t)w * lg.per;
    int i = threadIdx.x;
    for (; i + 3 * blockDim.x < n; i += 4 * blockDim.x) {
      uint32_t q[4];
      T val[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        q[k] = lg.cell[base + i + k * blockDim.x];
        val[k] = lg.val[base + i + k * blockDim.x];
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) vals[(size_t)(q[k] >> 9) * BV + (q[k] & 511)] = val[k];
      if (lo) {
#pragma unroll
        for (int k = 0; k < 4; ++k) lo[(size_t)(q[k] >> 9) * BV + (q[k] & 511)] = 0.f;
      }
    }
    for (; i < n; i += blockDim.x) {
      const uint32_t q = lg.cell[base + i];
      vals[(size_t)(q >> 9) * BV + (q & 511)] = lg.val[base + i];
      if (lo) lo[(size_t)(q >> 9) * BV + (q & 511)] = 0.f;
    }
    // the point data the pass logged with each value
    if (pd.src && lg.pd.src)
      for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const uint32_t q = lg.cell[base + j];
        const size_t c = (size_t)(q >> 9) * BV + (q & 511);
        pd.src[c] = lg.pd.src[base + j];
        pd.vel[c] = lg.pd.vel[base + j];
        pd.diss[c] = lg.pd.diss[base + j];
      }
  }
}

// Value of a cell after Reduce(1) + update: the (updated) value of an active
// cell, the sign sentinel of any other.  `actHere` holds the active planes of
// brick `slot` (shared memory); other bricks read `act`.
template <class T>
__device__ inline T reducedValue(const T *vals, const uint64_t *act, const unsigned long long *actHere,
                                 const int8_t *farSign, int slot, int ref, int loc) {
  if (ref < 0) return sentinel<T>(farSign[-1 - ref] < 0);
  const T val = vals[(size_t)ref * BV + loc];
  const uint64_t word = ref == slot ? actHere[loc >> 6] : act[(size_t)ref * 8 + (loc >> 6)];
  return ((word >> (loc & 63)) & 1ull) ? val : sentinel<T>(val < 0);
}

// rebuildLS after updateLevelSet (the active values are already updated in
// place): candidates are the active cells and their neighbours; every other
// defined cell becomes undefined with its sign.  Those cells are neither
// active nor candidates, so no evaluation in this pass reads more than their
// sign, which the sentinel keeps: they are rewritten in place, and only the
// candidates' new values go through the change log.
template <class T>
__global__ void __launch_bounds__(FRONTIER_THREADS, VLSG_PASS_MIN_BLOCKS)
    kUpdateRebuild(Topo t, LsView<T> v, const uint64_t *act, double cutoff, ChangeLog<T> lg,
                   const uint8_t *visitIn, uint8_t *visitOut) {
  __shared__ WarpScratch sm[FRONTIER_THREADS / 32];
  WarpScratch &ws = sm[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nWarps = (gridDim.x * blockDim.x) >> 5;
  const int n = *t.nSlots;
  const size_t logBase = (size_t)warp * lg.per;
  int logged = 0;
  const RebuildRule<T> rule{cutoff};
  for (int w = warp; w < n; w += nWarps) {
    const int slot = t.slotList[w];
    const bool complex = (t.cflag[slot] & CF_STAR) != 0;
    // a brick the previous pass of this buffer did not mark has no defined
    // cell (so no active one) and no defined face neighbour cell
    if (visitIn && !complex && !visitIn[slot]) {
      if (lane < 8) v.defNext[(size_t)slot * 8 + lane] = 0ull;
      continue;
    }
    if (lane < 8) ws.aux[lane] = act[(size_t)slot * 8 + lane];
    beginBrick(t, ws, slot, lane);
    int x0 = 0, y0 = 0, z0 = 0;
    if (complex) brickOrigin(t, slot, x0, y0, z0);
    const uint64_t own = lane < 8 ? v.def[(size_t)slot * 8 + lane] : 0ull;
    uint64_t cand;
    if (complex) cand = lane < 8 ? existPlane(t.g, x0, y0, z0, lane) : 0ull;
    else cand = dilatedMask(t, act, slot, ws.nb, lane);
    const uint64_t clear = own & ~cand;
    const int total = listCells(cand, ws.list);
    for (int base = 0; base < total; base += 32) {
      const int k = base + lane;
      bool changed = false;
      T out = T(0);
      int c = 0;
      int32_t ps = -1;
      T pv = T(0), pdi = T(0);
      if (k < total) {
        c = ws.list[k];
        const T mem = v.vals[(size_t)slot * BV + c];
        const T center = ((ws.aux[c >> 6] >> (c & 63)) & 1ull) ? mem : sentinel<T>(mem < 0);
        T nb[6];
#pragma unroll
        for (int j = 0; j < 6; ++j) {
          int loc;
          const int ref = starRef(t, ws.nb, slot, complex, x0, y0, z0, c, j, loc);
          nb[j] = reducedValue<T>(v.vals, act, ws.aux, v.farSign, slot, ref, loc);
        }
        int src = -1;
        out = rule(center, nb, src);
        changed = out != mem || signbit(out) != signbit(mem);
        if (changed && isDef(out) != isDef(mem)) markCell(ws.flip, c);
        if (lg.pd.src && isDef(out) && src >= 0) changed = true;
        if (changed && lg.pd.src && isDef(out)) {
          int loc = 0, ref = -1;
          if (src >= 0) ref = starRef(t, ws.nb, slot, complex, x0, y0, z0, c, src, loc);
          payloadOf<T>(v.pd, (size_t)slot * BV + c, src, ref, loc, ps, pv, pdi);
        }
      }
      logChange<T>(lg, logBase, logged, changed, ((uint32_t)slot << 9) | (uint32_t)c, out, ps,
                   pv, pdi);
    }
    // defined cells away from the active ones: undefined with their sign,
    // written in place (32 consecutive cells per step)
    __syncwarp();
    if (lane < 8) ws.aux[lane] = clear;
    __syncwarp();
    T *bv = v.vals + (size_t)slot * BV;
#pragma unroll 2
    for (int i = 0; i < 16; ++i) {
      const uint64_t word = ws.aux[i >> 1];
      if (!word) continue;
      const int c = i * 32 + lane;
      if ((word >> (c & 63)) & 1ull) bv[c] = sentinel<T>(bv[c] < 0);
    }
    __syncwarp();
    if (lane < 8) ws.flip[lane] |= clear;
    finishBrick(ws, v.defNext, slot, lane, own, visitOut);
  }
  if (lane == 0) lg.count[warp] = logged;
}

// Pointwise boolean of two level sets, in place on A (booleanOpInternal,
// lsBooleanOperation.hpp:100-132); rewrites A's current masks.  `flag` is
// set when the comparator reports a move (combineLevelSets).
template <class T, class Comp>
__global__ void __launch_bounds__(FRONTIER_THREADS)
    kPointwise(Topo t, T *av, uint64_t *adef, const T *bv, Comp comp, int *flag, float *alo) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nWarps = (gridDim.x * blockDim.x) >> 5;
  const int n = *t.nSlots;
  for (int w = warp; w < n; w += nWarps) {
    const int slot = t.slotList[w];
    int bx, by, bz;
    brickCoords(t.g, t.slotBrick[slot], bx, by, bz);
    const int x0 = t.g.org[0] + bx * BS, y0 = t.g.org[1] + by * BS, z0 = t.g.org[2] + bz * BS;
    bool moved = false;
    uint64_t mine = 0;
    for (int z = 0; z < 8; ++z) {
      uint64_t bits = 0;
      for (int half = 0; half < 2; ++half) {
        const int c = z * 64 + half * 32 + lane;
        const size_t q = (size_t)slot * BV + c;
        const T a = av[q], bb = bv[q];
        bool mv = false;
        T o = comp(a, bb, mv);
        if (!cellExists(t.g, x0 + (c & 7), y0 + ((c >> 3) & 7), z0 + (c >> 6))) {
          o = Lim<T>::max();
          mv = false;
        }
        moved |= mv;
        if (o != a || signbit(o) != signbit(a)) {
          av[q] = o;
          if (alo) alo[q] = 0.f;
        }
        bits |= (uint64_t)__ballot_sync(0xffffffffu, isDef(o)) << (32 * half);
      }
      if (lane == z) mine = bits;
    }
    if (lane < 8) adef[(size_t)slot * 8 + lane] = mine;
    if (__any_sync(0xffffffffu, moved) && lane == 0 && flag) atomicOr(flag, 1);
  }
}

// Pointwise boolean for comparators that keep every undefined cell of A
// (combineLevelSets, lsAdvect.hpp:218-230): only A's defined cells are read,
// in place; A's masks lose the cells that became undefined.
// With compensation terms of both (FP32 buffers: alo for A, blo for B) the
// comparator sees hi + lo of each value in double and the result is split
// again into hi and lo (Comp::full); with alo alone a changed value's term
// becomes 0.
template <class T, class Comp>
__global__ void __launch_bounds__(FRONTIER_THREADS)
    kPointwiseDefined(Topo t, T *av, uint64_t *adef, const T *bv, Comp comp, int *flag,
                      float *alo, const float *blo) {
  __shared__ WarpScratch sm[FRONTIER_THREADS / 32];
  WarpScratch &ws = sm[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nWarps = (gridDim.x * blockDim.x) >> 5;
  const int n = *t.nSlots;
  bool moved = false;
  for (int w = warp; w < n; w += nWarps) {
    const int slot = t.slotList[w];
    const uint64_t own = lane < 8 ? adef[(size_t)slot * 8 + lane] : 0ull;
    if (!__any_sync(0xffffffffu, own != 0ull)) continue;
    if (lane < 8) ws.flip[lane] = 0ull;
    const int total = listCells(own, ws.list);
    for (int base = 0; base < total; base += 32) {
      const int k = base + lane;
      if (k >= total) continue;
      const int c = ws.list[k];
      const size_t q = (size_t)slot * BV + c;
      const T a = av[q];
      bool mv = false;
      if constexpr (sizeof(T) == 4) {
        if (alo && blo) {
          const T b = bv[q];
          if (isDef(b)) {
            const double r = comp.full(withLo((double)a, alo[q]), withLo((double)b, blo[q]), mv);
            const float hi = (float)r;
            av[q] = hi;
            alo[q] = (float)(r - (double)hi);
          } else {
            av[q] = b;
            markCell(ws.flip, c);
          }
          moved |= mv;
          continue;
        }
      }
      const T o = comp(a, bv[q], mv);
      moved |= mv;
      if (o != a || signbit(o) != signbit(a)) {
        av[q] = o;
        if (alo) alo[q] = 0.f;
        if (!isDef(o)) markCell(ws.flip, c);
      }
    }
    __syncwarp();
    if (lane < 8) adef[(size_t)slot * 8 + lane] = own & ~ws.flip[lane];
    __syncwarp();
  }
  if (__any_sync(0xffffffffu, moved) && lane == 0 && flag) atomicOr(flag, 1);
}

// Copy the listed slots of one buffer (values and masks) into another, 16
// bytes per thread.
// dlo (a compensation array of the destination, or null) receives slo, or
// zeros when the source has none.
template <class T>
__global__ void kCopySlots16(const int *slotList, const int *nSlots, const T *sv,
                             const uint64_t *sd, T *dv, uint64_t *dd, const float *slo,
                             float *dlo) {
  constexpr int PER = BV * sizeof(T) / 16; // 16-byte words per slot
  const size_t n = (size_t)*nSlots * PER;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const size_t slot = slotList[i / PER];
    const int k = (int)(i % PER);
    reinterpret_cast<uint4 *>(dv + slot * BV)[k] = reinterpret_cast<const uint4 *>(sv + slot * BV)[k];
    if (k < 4) reinterpret_cast<uint4 *>(dd + slot * 8)[k] = reinterpret_cast<const uint4 *>(sd + slot * 8)[k];
    if (dlo && k < BV * 4 / 16) {
      const uint4 z = make_uint4(0u, 0u, 0u, 0u);
      reinterpret_cast<uint4 *>(dlo + slot * BV)[k] =
          slo ? reinterpret_cast<const uint4 *>(slo + slot * BV)[k] : z;
    }
  }
}

// Neighbour table and complexity flags of every listed slot, for any
// boundary conditions: entry = slot, or -1-brick (unallocated, or outside the
// map box: the nearest box brick).  CF_STAR: the brick holds a cell whose
// star neighbour is remapped by a boundary (or a cell past the grid's end);
// CF_NEAR: such a cell lies within 8 cells of the brick.
__device__ inline bool remapNear(const GridDev &g, int d, int lo, int hi) {
  switch (g.bc[d]) {
  case VLSG_PERIODIC_BOUNDARY:
    return (g.gmax[d] - g.gmin[d]) % BS != 0 && (lo <= g.gmin[d] || hi >= g.gmax[d] - 1);
  case VLSG_REFLECTIVE_BOUNDARY:
    return lo <= g.gmin[d] || hi >= g.gmax[d];
  case VLSG_POS_INFINITE_BOUNDARY:
    return lo <= g.gmin[d];
  case VLSG_NEG_INFINITE_BOUNDARY:
    return hi >= g.gmax[d];
  default:
    return false;
  }
}

__global__ void kBuildNeighbours(GridDev g, const int *brickMap, const int *slotBrick,
                                 const int *slotList, const int *nSlots, int *nbr,
                                 uint8_t *cflag, int *slotDom) {
  const int n = *nSlots;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int slot = slotList[i];
    int bx, by, bz;
    brickCoords(g, slotBrick[slot], bx, by, bz);
    if (g.nDom) {
      // batching form: wrap within the brick's domain; a neighbour past the
      // domain's brick planes is the nearest plane's (unallocated) brick
      const int d = g.domOfBz[bz];
      slotDom[slot] = d;
      cflag[slot] = 0;
      for (int k = 0; k < 27; ++k) {
        int x = bx + k % 3 - 1, y = by + (k / 3) % 3 - 1, z = bz + k / 9 - 1;
        const bool inside = domainNeighbour(g, d, x, y, z);
        if (!inside) z = z < g.dom[d].bz0 ? g.dom[d].bz0 : g.dom[d].bz1 - 1;
        const int bi = brickIndex(g, x, y, z);
        const int s = brickMap[bi];
        nbr[(size_t)slot * 27 + k] = (s >= 0 && inside) ? s : -1 - bi;
      }
      continue;
    }
    const int bc[3] = {bx, by, bz};
    uint8_t f = 0;
    for (int d = 0; d < 3; ++d) {
      const int lo = g.org[d] + bc[d] * BS, hi = lo + BS - 1;
      if (remapNear(g, d, lo, hi)) f |= CF_STAR | CF_NEAR;
      if (remapNear(g, d, lo - BS, hi + BS)) f |= CF_NEAR;
    }
    cflag[slot] = f;
    for (int k = 0; k < 27; ++k) {
      int c[3] = {bx + k % 3 - 1, by + (k / 3) % 3 - 1, bz + k / 9 - 1};
      bool outside = false;
      for (int d = 0; d < 3; ++d) {
        if (c[d] >= 0 && c[d] < g.nb[d]) continue;
        if (g.bc[d] == VLSG_PERIODIC_BOUNDARY) {
          c[d] = (c[d] + g.nb[d]) % g.nb[d];
        } else {
          c[d] = c[d] < 0 ? 0 : g.nb[d] - 1;
          outside = true;
        }
      }
      const int bi = brickIndex(g, c[0], c[1], c[2]);
      const int s = brickMap[bi];
      nbr[(size_t)slot * 27 + k] = (s >= 0 && !outside) ? s : -1 - bi;
    }
  }
}

} // namespace
} // namespace vlsg
