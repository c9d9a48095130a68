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

template <class T> struct LsView {
  T *vals;               // slots x 512 cells, in place
  const uint64_t *def;   // current masks, slots x 8 words
  uint64_t *defNext;     // masks after the pass
  const int8_t *farSign; // per brick of the map box
};

// Change log: segment w (of `per` entries) belongs to warp w of the pass.
template <class T> struct ChangeLog {
  uint32_t *cell; // slot << 9 | cell
  T *val;
  int *count;     // entries per segment
  size_t per;
};

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

// Per-warp context of one brick.
struct BrickCtx {
  int slot, nb[6]; // face neighbours -x,+x,-y,+y,-z,+z (slot or -1-brick)
  bool complex;
  int x0, y0, z0;
};

__device__ inline BrickCtx loadBrickCtx(const Topo &t, int slot) {
  BrickCtx b;
  b.slot = slot;
  const int *n = t.nbr + (size_t)slot * 27;
  b.nb[0] = n[NB_XM], b.nb[1] = n[NB_XP], b.nb[2] = n[NB_YM];
  b.nb[3] = n[NB_YP], b.nb[4] = n[NB_ZM], b.nb[5] = n[NB_ZP];
  b.complex = (t.cflag[slot] & CF_STAR) != 0;
  int bx, by, bz;
  brickCoords(t.g, t.slotBrick[slot], bx, by, bz);
  b.x0 = t.g.org[0] + bx * BS, b.y0 = t.g.org[1] + by * BS, b.z0 = t.g.org[2] + bz * BS;
  return b;
}

// Star neighbours (order +x,+y,+z,-x,-y,-z) of local cell c as (slot or
// -1-brick, cell) pairs.
__device__ inline void starRefs(const Topo &t, const BrickCtx &b, int c, int *ref, int *loc) {
  const int x = c & 7, y = (c >> 3) & 7, z = c >> 6;
  if (b.complex) {
    const int X = b.x0 + x, Y = b.y0 + y, Z = b.z0 + z;
    ref[0] = locateCell(t.g, t.brickMap, X + 1, Y, Z, loc[0]);
    ref[1] = locateCell(t.g, t.brickMap, X, Y + 1, Z, loc[1]);
    ref[2] = locateCell(t.g, t.brickMap, X, Y, Z + 1, loc[2]);
    ref[3] = locateCell(t.g, t.brickMap, X - 1, Y, Z, loc[3]);
    ref[4] = locateCell(t.g, t.brickMap, X, Y - 1, Z, loc[4]);
    ref[5] = locateCell(t.g, t.brickMap, X, Y, Z - 1, loc[5]);
    return;
  }
  ref[0] = x < 7 ? b.slot : b.nb[1], loc[0] = x < 7 ? c + 1 : c - 7;
  ref[1] = y < 7 ? b.slot : b.nb[3], loc[1] = y < 7 ? c + 8 : c - 56;
  ref[2] = z < 7 ? b.slot : b.nb[5], loc[2] = z < 7 ? c + 64 : c - 448;
  ref[3] = x > 0 ? b.slot : b.nb[0], loc[3] = x > 0 ? c - 1 : c + 7;
  ref[4] = y > 0 ? b.slot : b.nb[2], loc[4] = y > 0 ? c - 8 : c + 56;
  ref[5] = z > 0 ? b.slot : b.nb[4], loc[5] = z > 0 ? c - 64 : c + 448;
}

template <class T>
__device__ inline T refValue(const T *vals, const int8_t *farSign, int ref, int loc) {
  return ref >= 0 ? vals[(size_t)ref * BV + loc] : sentinel<T>(farSign[-1 - ref] < 0);
}

// Mask of the cells of plane z that exist in the grid.
__device__ inline uint64_t existPlane(const GridDev &g, const BrickCtx &b, int z) {
  uint64_t m = 0;
  for (int y = 0; y < 8; ++y)
    for (int x = 0; x < 8; ++x)
      if (cellExists(g, b.x0 + x, b.y0 + y, b.z0 + z)) m |= 1ull << (y * 8 + x);
  return m;
}

// Star dilation of the brick's mask, plane of lane z (lanes 0..7; the other
// lanes return 0).  Every lane of the warp must call it.  Sets err bit 64
// when a set cell lies on a face whose neighbour brick is not allocated
// (its cells could change but are not in the pool).
__device__ inline uint64_t dilatedMask(const Topo &t, const uint64_t *mask, const BrickCtx &b,
                                       int lane) {
  const int z = lane & 7;
  const uint64_t w = lane < 8 ? mask[(size_t)b.slot * 8 + z] : 0ull;
  uint64_t below = __shfl_sync(0xffffffffu, w, (z + 7) & 7);
  uint64_t above = __shfl_sync(0xffffffffu, w, (z + 1) & 7);
  if (lane >= 8) return 0ull;
  if (z == 0) below = b.nb[4] >= 0 ? mask[(size_t)b.nb[4] * 8 + 7] : 0ull;
  if (z == 7) above = b.nb[5] >= 0 ? mask[(size_t)b.nb[5] * 8 + 0] : 0ull;
  const uint64_t nxm = b.nb[0] >= 0 ? mask[(size_t)b.nb[0] * 8 + z] : 0ull;
  const uint64_t nxp = b.nb[1] >= 0 ? mask[(size_t)b.nb[1] * 8 + z] : 0ull;
  const uint64_t nym = b.nb[2] >= 0 ? mask[(size_t)b.nb[2] * 8 + z] : 0ull;
  const uint64_t nyp = b.nb[3] >= 0 ? mask[(size_t)b.nb[3] * 8 + z] : 0ull;
  const bool open = ((w & XLO) && b.nb[0] < 0) || ((w & XHI) && b.nb[1] < 0) ||
                    ((w & 0xffull) && b.nb[2] < 0) || ((w >> 56) && b.nb[3] < 0) ||
                    (z == 0 && w && b.nb[4] < 0) || (z == 7 && w && b.nb[5] < 0);
  if (open) atomicOr(t.err, 64);
  return w | ((w << 1) & ~XLO) | ((w >> 1) & ~XHI) | ((nxm & XHI) >> 7) | ((nxp & XLO) << 7) |
         (w << 8) | (w >> 8) | (nym >> 56) | (nyp << 56) | below | above;
}

// Enumeration of the set bits of a 512-bit brick mask held as one plane word
// per lane 0..7 (lane z: plane z): the k-th set bit in (z, y, x) order, so a
// warp takes 32 cells of the brick per round whatever planes they lie in.
// Every lane of the warp must construct it and call cell().
struct PlaneEnum {
  int incl[8]; // inclusive prefix counts over the planes (in every lane)
  int total;
  __device__ explicit PlaneEnum(uint64_t w) {
    const int lane = threadIdx.x & 31;
    int cnt = lane < 8 ? __popcll(w) : 0;
#pragma unroll
    for (int o = 1; o < 8; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, cnt, o, 8);
      if ((lane & 7) >= o) cnt += t;
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) incl[j] = __shfl_sync(0xffffffffu, cnt, j);
    total = incl[7];
  }
  // Cell index z*64+y*8+x of set bit k (k clamped into range by the caller).
  __device__ int cell(uint64_t w, int k) const {
    int z = 0, excl = 0;
#pragma unroll
    for (int j = 0; j < 7; ++j)
      if (k >= incl[j]) z = j + 1, excl = incl[j];
    const uint64_t m = __shfl_sync(0xffffffffu, w, z);
    const unsigned lo = (unsigned)m, hi = (unsigned)(m >> 32);
    const int nlo = __popc(lo), r = k - excl;
    const int bit = r < nlo ? (int)__fns(lo, 0, r + 1) : 32 + (int)__fns(hi, 0, r - nlo + 1);
    return z * 64 + bit;
  }
};

// Per-warp shared words of the brick in hand: cells whose definedness flips.
struct WarpMasks {
  unsigned long long flip[8];
};

__device__ inline void markCell(unsigned long long *words, int c) {
  atomicOr(&words[c >> 6], 1ull << (c & 63));
}

// Publish the brick's new defined mask (old ^ flips).
__device__ inline void finishBrick(WarpMasks &m, uint64_t *defNext, int slot, int lane,
                                   uint64_t own) {
  __syncwarp();
  if (lane < 8) defNext[(size_t)slot * 8 + lane] = own ^ m.flip[lane];
  __syncwarp();
}

__device__ inline void clearBrick(WarpMasks &m, int lane) {
  if (lane < 8) m.flip[lane] = 0ull;
  __syncwarp();
}

// Append the lanes with `has` to the warp's log segment (warp-uniform call).
template <class T>
__device__ inline void logChange(const ChangeLog<T> &lg, size_t base, int &count, bool has,
                                 uint32_t cell, T val) {
  const unsigned m = __ballot_sync(0xffffffffu, has);
  if (has) {
    const size_t p = base + count + __popc(m & ((1u << (threadIdx.x & 31)) - 1));
    lg.cell[p] = cell;
    lg.val[p] = val;
  }
  count += __popc(m);
}

enum : int { FP_EXPAND = 0, FP_PRUNE = 1, FP_ALL = 2 };

// One star pass of a rule.  MODE picks the candidates: FP_EXPAND undefined
// cells next to a defined one, FP_PRUNE the defined cells, FP_ALL the
// defined cells and their neighbours.
template <class T, int MODE, class Rule>
__global__ void __launch_bounds__(FRONTIER_THREADS, VLSG_PASS_MIN_BLOCKS)
    kFrontierPass(Topo t, LsView<T> v, Rule rule, ChangeLog<T> lg) {
  __shared__ WarpMasks sm[FRONTIER_THREADS / 32];
  WarpMasks &wm = sm[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nWarps = (gridDim.x * blockDim.x) >> 5;
  const int n = *t.nSlots;
  const size_t logBase = (size_t)warp * lg.per;
  int logged = 0;
  for (int w = warp; w < n; w += nWarps) {
    const int slot = t.slotList[w];
    const BrickCtx b = loadBrickCtx(t, slot);
    const uint64_t own = lane < 8 ? v.def[(size_t)slot * 8 + lane] : 0ull;
    uint64_t cand;
    if (MODE == FP_PRUNE) {
      cand = own;
    } else if (b.complex) {
      const uint64_t ex = lane < 8 ? existPlane(t.g, b, lane) : 0ull;
      cand = MODE == FP_EXPAND ? ex & ~own : ex;
    } else {
      const uint64_t dil = dilatedMask(t, v.def, b, lane);
      cand = MODE == FP_EXPAND ? dil & ~own : dil;
    }
    clearBrick(wm, lane);
    const PlaneEnum pe(cand);
    for (int base = 0; base < pe.total; base += 32) {
      const int k = base + lane;
      const int c = pe.cell(cand, k < pe.total ? k : pe.total - 1);
      bool changed = false;
      T out = T(0);
      if (k < pe.total) {
        const size_t q = (size_t)slot * BV + c;
        const T center = v.vals[q];
        int ref[6], loc[6];
        starRefs(t, b, c, ref, loc);
        T nb[6];
#pragma unroll
        for (int j = 0; j < 6; ++j) nb[j] = refValue<T>(v.vals, v.farSign, ref[j], loc[j]);
        out = rule(center, nb);
        changed = out != center || signbit(out) != signbit(center);
        if (changed && isDef(out) != isDef(center)) markCell(wm.flip, c);
      }
      logChange<T>(lg, logBase, logged, changed, ((uint32_t)slot << 9) | (uint32_t)c, out);
    }
    finishBrick(wm, v.defNext, slot, lane, own);
  }
  if (lane == 0) lg.count[warp] = logged;
}

// Write a change log back: warp w copies segment w.
template <class T>
__global__ void __launch_bounds__(FRONTIER_THREADS)
    kApplyChanges(T *vals, ChangeLog<T> lg, int segments) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nWarps = (gridDim.x * blockDim.x) >> 5;
  for (int w = warp; w < segments; w += nWarps) {
    const int n = lg.count[w];
    const size_t base = (size_t)w * lg.per;
    for (int i = lane; i < n; i += 32) {
      const uint32_t q = lg.cell[base + i];
      vals[(size_t)(q >> 9) * BV + (q & 511)] = lg.val[base + i];
    }
  }
}

// Value of a cell after Reduce(1) + update: the (updated) value of an active
// cell, the sign sentinel of any other.
template <class T>
__device__ inline T reducedValue(const T *vals, const uint64_t *act, const int8_t *farSign,
                                 int ref, int loc) {
  if (ref < 0) return sentinel<T>(farSign[-1 - ref] < 0);
  const T val = vals[(size_t)ref * BV + loc];
  const bool a = (act[(size_t)ref * 8 + (loc >> 6)] >> (loc & 63)) & 1ull;
  return a ? val : sentinel<T>(val < 0);
}

// rebuildLS after updateLevelSet (the active values are already updated in
// place): candidates are the active cells and their neighbours; every other
// defined cell becomes undefined with its sign.
template <class T>
__global__ void __launch_bounds__(FRONTIER_THREADS, VLSG_PASS_MIN_BLOCKS)
    kUpdateRebuild(Topo t, LsView<T> v, const uint64_t *act, double cutoff, ChangeLog<T> lg) {
  __shared__ WarpMasks sm[FRONTIER_THREADS / 32];
  WarpMasks &wm = sm[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nWarps = (gridDim.x * blockDim.x) >> 5;
  const int n = *t.nSlots;
  const size_t logBase = (size_t)warp * lg.per;
  int logged = 0;
  const RebuildRule<T> rule{cutoff};
  for (int w = warp; w < n; w += nWarps) {
    const int slot = t.slotList[w];
    const BrickCtx b = loadBrickCtx(t, slot);
    const uint64_t own = lane < 8 ? v.def[(size_t)slot * 8 + lane] : 0ull;
    uint64_t cand;
    if (b.complex) cand = lane < 8 ? existPlane(t.g, b, lane) : 0ull;
    else cand = dilatedMask(t, act, b, lane);
    const uint64_t clear = own & ~cand;
    clearBrick(wm, lane);
    const PlaneEnum pe(cand);
    for (int base = 0; base < pe.total; base += 32) {
      const int k = base + lane;
      const int c = pe.cell(cand, k < pe.total ? k : pe.total - 1);
      bool changed = false;
      T out = T(0);
      if (k < pe.total) {
        const size_t q = (size_t)slot * BV + c;
        const T mem = v.vals[q];
        const T center = reducedValue<T>(v.vals, act, v.farSign, slot, c);
        int ref[6], loc[6];
        starRefs(t, b, c, ref, loc);
        T nb[6];
#pragma unroll
        for (int j = 0; j < 6; ++j) nb[j] = reducedValue<T>(v.vals, act, v.farSign, ref[j], loc[j]);
        out = rule(center, nb);
        changed = out != mem || signbit(out) != signbit(mem);
        if (changed && isDef(out) != isDef(mem)) markCell(wm.flip, c);
      }
      logChange<T>(lg, logBase, logged, changed, ((uint32_t)slot << 9) | (uint32_t)c, out);
    }
    // defined cells away from the active ones: undefined with their sign
    const PlaneEnum pc(clear);
    for (int base = 0; base < pc.total; base += 32) {
      const int k = base + lane;
      const int c = pc.cell(clear, k < pc.total ? k : pc.total - 1);
      T out = T(0);
      if (k < pc.total) out = sentinel<T>(v.vals[(size_t)slot * BV + c] < 0);
      logChange<T>(lg, logBase, logged, k < pc.total, ((uint32_t)slot << 9) | (uint32_t)c, out);
    }
    __syncwarp();
    if (lane < 8) wm.flip[lane] |= clear;
    finishBrick(wm, v.defNext, slot, lane, own);
  }
  if (lane == 0) lg.count[warp] = logged;
}

// Pointwise boolean of two level sets, in place on A (booleanOpInternal,
// lsBooleanOperation.hpp:100-132); rewrites A's current masks.  `flag` is
// set when the comparator reports a move (combineLevelSets).
template <class T, class Comp>
__global__ void __launch_bounds__(FRONTIER_THREADS)
    kPointwise(Topo t, T *av, uint64_t *adef, const T *bv, Comp comp, int *flag) {
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
        if (o != a || signbit(o) != signbit(a)) av[q] = o;
        bits |= (uint64_t)__ballot_sync(0xffffffffu, isDef(o)) << (32 * half);
      }
      if (lane == z) mine = bits;
    }
    if (lane < 8) adef[(size_t)slot * 8 + lane] = mine;
    if (__any_sync(0xffffffffu, moved) && lane == 0 && flag) atomicOr(flag, 1);
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
                                 uint8_t *cflag) {
  const int n = *nSlots;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int slot = slotList[i];
    int bx, by, bz;
    brickCoords(g, slotBrick[slot], bx, by, bz);
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
