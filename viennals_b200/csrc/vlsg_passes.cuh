// vlsg_passes.cuh -- band-maintenance passes of libvlsgpu as brick stencils.
//
// Every rule below is a pointwise function of a cell and its six star
// neighbours, restated from the reference:
//   ExpandRule   Expand::apply            lsExpand.hpp:104-157
//   PruneRule    Prune::apply             lsPrune.hpp:118-180
//   RebuildRule  Advect::rebuildLS        lsAdvect.hpp:299-415
// and pointwise rules of two level sets:
//   booleanOpInternal + comparators       lsBooleanOperation.hpp:100-132, :262-280
//   combineLevelSets comparator           lsAdvect.hpp:218-230
// Neighbour order is the reference star iterator's: +x,+y,+z,-x,-y,-z.
//
// One CTA of 256 threads handles one 8^3 brick per iteration of a grid-stride
// loop over the slot list: the brick and its six face layers are staged in
// shared memory as a 10^3 box (faces read through the brick map, so periodic
// and reflective boundaries need no special case), every thread evaluates two
// cells, and a block vote decides whether the output brick is DENSE or
// UNIFORM (then no cell is written).
#pragma once

#include "vlsg_common.cuh"

namespace vlsg {

constexpr int PASS_THREADS = 256;

template <class T> struct ExpandRule {
  T totalLimit, limit;
  __device__ T operator()(T c, const T *nb) const {
    if (fabs(c) <= totalLimit) return c;
    if (c > -Lim<T>::eps()) {
      T distance = Lim<T>::max();
      for (int i = 0; i < 6; ++i) {
        const T nv = nb[i] + T(1);
        if (distance > nv) distance = nv;
      }
      return distance <= limit ? distance : Lim<T>::max();
    }
    T distance = Lim<T>::lowest();
    for (int i = 0; i < 6; ++i) {
      const T nv = nb[i] - T(1);
      if (distance < nv) distance = nv;
    }
    return distance >= -limit ? distance : Lim<T>::lowest();
  }
};

template <class T> struct PruneRule {
  bool removeStrayZeros;
  __device__ static bool neg(T a) { return a <= -Lim<T>::eps(); }
  __device__ static bool diff(T a, T b) { return neg(a) != neg(b); }
  __device__ T operator()(T c, const T *nb) const {
    const bool cneg = neg(c);
    if (!isDef(c)) return cneg ? Lim<T>::lowest() : Lim<T>::max();
    bool keep = true;
    if (fabs(c) != T(0)) {
      keep = false;
      for (int i = 0; i < 6; ++i) {
        const bool d = removeStrayZeros ? (c == T(0) || nb[i] == T(0) || diff(c, nb[i]))
                                        : diff(c, nb[i]);
        if (d) {
          keep = true;
          break;
        }
      }
    }
    if (removeStrayZeros && fabs(c) == T(0)) {
      for (int i = 0; i < 3; ++i) {
        const T a = nb[i], b = nb[3 + i];
        const bool monotone = a == T(0) || b == T(0) || diff(a, b);
        if (!monotone) return fabs(a) < fabs(b) ? a : b;
      }
    }
    if (keep) return c;
    return cneg ? Lim<T>::lowest() : Lim<T>::max();
  }
};

template <class T> struct RebuildRule {
  double cutoff;
  __device__ T operator()(T cT, const T *nb) const {
    const double c = (double)cT;
    if (fabs(c) <= 1.0) {
      int k = 0;
      for (; k < 6; k++)
        if (signbit((double)nb[k] - 1e-7) != signbit(c + 1e-7)) break;
      if (k != 6) {
        if (c > 0.5) {
          int j = 0;
          for (; j < 6; j++)
            if (fabs((double)nb[j]) <= 1.0 && (double)nb[j] < -0.5) break;
          return j == 6 ? cT : T(0.5);
        } else if (c < -0.5) {
          int j = 0;
          for (; j < 6; j++)
            if (fabs((double)nb[j]) <= 1.0 && (double)nb[j] > 0.5) break;
          return j == 6 ? cT : T(-0.5);
        }
        return cT;
      }
      return c < 0 ? Lim<T>::lowest() : Lim<T>::max();
    }
    if (c >= 0) {
      T distance = Lim<T>::max();
      for (int i = 0; i < 6; i++) {
        const double v = (double)nb[i];
        if (fabs(v) <= 1.0 && (v < 0.))
          if ((double)distance > v + 1.0) distance = T(v + 1.0);
      }
      return (double)distance <= cutoff ? distance : Lim<T>::max();
    }
    T distance = Lim<T>::lowest();
    for (int i = 0; i < 6; i++) {
      const double v = (double)nb[i];
      if (fabs(v) <= 1.0 && (v > 0))
        if ((double)distance < v - 1.0) distance = T(v - 1.0);
    }
    return (double)distance >= -cutoff ? distance : Lim<T>::lowest();
  }
};

// Pass arguments shared by the brick kernels.
template <class T> struct PassOut {
  T *vals;
  uint8_t *state;
  uint8_t *hasDef;
  unsigned long long *defCount; // defined output cells (for byte accounting)
};

// Add the block's defined output cells (two per thread) to *cnt.
template <class T>
__device__ inline void countDefined(const T *res, unsigned long long *cnt) {
  const int nd = __syncthreads_count(isDef(res[0])) + __syncthreads_count(isDef(res[1]));
  if (threadIdx.x == 0 && cnt && nd) atomicAdd(cnt, (unsigned long long)nd);
}

// Box of 10^3 cells around a brick in shared memory.
__device__ inline int boxIdx(int x, int y, int z) {
  return ((z + 1) * 10 + (y + 1)) * 10 + (x + 1);
}

// Sign of the brick adjacent through face f (0..5 = -x,+x,-y,+y,-z,+z) when
// it is uniform or unallocated; 0 when it is dense or cannot be decided at
// brick level (boundaries that remap cells inside a brick).
template <class T>
__device__ inline int faceNeighbourSign(const GridDev &g, const MapView &m,
                                        const Buf<T> &b, int bx, int by, int bz,
                                        int f) {
  int c[3] = {bx, by, bz};
  const int d = f >> 1;
  c[d] += (f & 1) ? 1 : -1;
  if (c[d] < 0 || c[d] >= g.nb[d]) {
    if (g.bc[d] == VLSG_INFINITE_BOUNDARY) {
      c[d] = c[d] < 0 ? 0 : g.nb[d] - 1;
    } else if (g.bc[d] == VLSG_PERIODIC_BOUNDARY &&
               ((g.gmax[d] - g.gmin[d]) % BS) == 0) {
      c[d] = (c[d] + g.nb[d]) % g.nb[d];
    } else {
      return 0;
    }
  }
  const int bi = brickIndex(g, c[0], c[1], c[2]);
  const int slot = m.brickMap[bi];
  if (slot < 0) return b.farSign[bi] < 0 ? -1 : 1;
  const uint8_t st = b.state[slot];
  if (st == ST_DENSE) return 0;
  return st == ST_UNEG ? -1 : 1;
}

// Generic star pass: out = rule(center, star neighbours) for every cell of
// every listed slot.
template <class T, class Rule>
__global__ void __launch_bounds__(PASS_THREADS)
    kStarPass(GridDev g, MapView m, const int *slotList, const int *nSlots,
              Buf<T> in, PassOut<T> out, Rule rule) {
  __shared__ T box[1000];
  __shared__ int skipSign;
  const int n = *nSlots;
  for (int it = blockIdx.x; it < n; it += gridDim.x) {
    const int slot = slotList[it];
    const int bi = m.slotBrick[slot];
    int bx, by, bz;
    brickCoords(g, bi, bx, by, bz);
    const int x0 = g.org[0] + bx * BS, y0 = g.org[1] + by * BS, z0 = g.org[2] + bz * BS;
    const uint8_t st = in.state[slot];
    if (threadIdx.x == 0) {
      int s = 0;
      if (st != ST_DENSE) {
        s = st == ST_UNEG ? -1 : 1;
        for (int f = 0; f < 6 && s != 0; ++f)
          if (faceNeighbourSign<T>(g, m, in, bx, by, bz, f) != s) s = 0;
      }
      skipSign = s;
    }
    __syncthreads();
    const int ss = skipSign;
    if (ss != 0) {
      // uniform brick in a uniform neighbourhood of the same sign: every rule
      // maps it to itself
      if (threadIdx.x == 0) {
        out.state[slot] = st;
        out.hasDef[slot] = 0;
      }
      __syncthreads();
      continue;
    }
    for (int c = threadIdx.x; c < BV; c += PASS_THREADS) {
      const int lx = c & 7, ly = (c >> 3) & 7, lz = c >> 6;
      T v;
      if (!cellExists(g, x0 + lx, y0 + ly, z0 + lz))
        // a cell past the end of a bounded direction stands for its image
        // under the boundary condition (the star neighbour of the last cell)
        v = cellValueRaw<T>(g, m, in, x0 + lx, y0 + ly, z0 + lz);
      else if (st == ST_DENSE) v = in.vals[(size_t)slot * BV + c];
      else v = st == ST_UNEG ? Lim<T>::lowest() : Lim<T>::max();
      box[boxIdx(lx, ly, lz)] = v;
    }
    for (int f = threadIdx.x; f < 384; f += PASS_THREADS) {
      const int face = f >> 6, a = f & 7, b2 = (f >> 3) & 7;
      int lx, ly, lz;
      const int d = face >> 1;
      const int side = (face & 1) ? BS : -1;
      if (d == 0) lx = side, ly = a, lz = b2;
      else if (d == 1) lx = a, ly = side, lz = b2;
      else lx = a, ly = b2, lz = side;
      box[boxIdx(lx, ly, lz)] = cellValueRaw<T>(g, m, in, x0 + lx, y0 + ly, z0 + lz);
    }
    __syncthreads();
    T res[2];
    bool anyDef = false, allPos = true, allNeg = true;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int c = threadIdx.x + k * PASS_THREADS;
      const int lx = c & 7, ly = (c >> 3) & 7, lz = c >> 6;
      const T center = box[boxIdx(lx, ly, lz)];
      T nb[6];
      nb[0] = box[boxIdx(lx + 1, ly, lz)];
      nb[1] = box[boxIdx(lx, ly + 1, lz)];
      nb[2] = box[boxIdx(lx, ly, lz + 1)];
      nb[3] = box[boxIdx(lx - 1, ly, lz)];
      nb[4] = box[boxIdx(lx, ly - 1, lz)];
      nb[5] = box[boxIdx(lx, ly, lz - 1)];
      T o = rule(center, nb);
      if (!cellExists(g, x0 + lx, y0 + ly, z0 + lz)) o = Lim<T>::max();
      else if (isDef(o)) anyDef = true;
      else if (o < 0) allPos = false;
      else allNeg = false;
      res[k] = o;
    }
    // phantom cells (beyond the end of a bounded direction) never count
    countDefined<T>(res, out.defCount);
    const int any = __syncthreads_or(anyDef);
    const int ap = __syncthreads_and(allPos);
    const int an = __syncthreads_and(allNeg);
    if (!any && (ap || an)) {
      if (threadIdx.x == 0) {
        out.state[slot] = ap ? ST_UPOS : ST_UNEG;
        out.hasDef[slot] = 0;
      }
    } else {
      if (!any && ap == 0 && an == 0) {
        // mixed-sign undefined brick: keep it dense
      }
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const int c = threadIdx.x + k * PASS_THREADS;
        out.vals[(size_t)slot * BV + c] = res[k];
      }
      if (threadIdx.x == 0) {
        out.state[slot] = ST_DENSE;
        out.hasDef[slot] = any ? 1 : 0;
      }
    }
    __syncthreads();
  }
}

// Pointwise pass of two level sets (boolean operations): out = comp(a, b).
template <class T, class Comp>
__global__ void __launch_bounds__(PASS_THREADS)
    kPointwise2(GridDev g, MapView m, const int *slotList, const int *nSlots,
                Buf<T> A, Buf<T> B, PassOut<T> out, Comp comp, int *flag) {
  const int n = *nSlots;
  for (int it = blockIdx.x; it < n; it += gridDim.x) {
    const int slot = slotList[it];
    const uint8_t sa = A.state[slot], sb = B.state[slot];
    const int bi = m.slotBrick[slot];
    int bx, by, bz;
    brickCoords(g, bi, bx, by, bz);
    const int x0 = g.org[0] + bx * BS, y0 = g.org[1] + by * BS, z0 = g.org[2] + bz * BS;
    T res[2];
    bool anyDef = false, allPos = true, allNeg = true, moved = false;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int c = threadIdx.x + k * PASS_THREADS;
      const T a = sa == ST_DENSE ? A.vals[(size_t)slot * BV + c]
                                 : (sa == ST_UNEG ? Lim<T>::lowest() : Lim<T>::max());
      const T b = sb == ST_DENSE ? B.vals[(size_t)slot * BV + c]
                                 : (sb == ST_UNEG ? Lim<T>::lowest() : Lim<T>::max());
      bool mv = false;
      T o = comp(a, b, mv);
      const int lx = c & 7, ly = (c >> 3) & 7, lz = c >> 6;
      if (!cellExists(g, x0 + lx, y0 + ly, z0 + lz)) o = Lim<T>::max(), mv = false;
      else if (isDef(o)) anyDef = true;
      else if (o < 0) allPos = false;
      else allNeg = false;
      moved |= mv;
      res[k] = o;
    }
    countDefined<T>(res, out.defCount);
    const int any = __syncthreads_or(anyDef);
    const int ap = __syncthreads_and(allPos);
    const int an = __syncthreads_and(allNeg);
    const int mvAny = __syncthreads_or(moved);
    if (threadIdx.x == 0 && mvAny && flag) atomicOr(flag, 1);
    if (!any && (ap || an)) {
      if (threadIdx.x == 0) {
        out.state[slot] = ap ? ST_UPOS : ST_UNEG;
        out.hasDef[slot] = 0;
      }
    } else {
#pragma unroll
      for (int k = 0; k < 2; ++k)
        out.vals[(size_t)slot * BV + threadIdx.x + k * PASS_THREADS] = res[k];
      if (threadIdx.x == 0) {
        out.state[slot] = ST_DENSE;
        out.hasDef[slot] = any ? 1 : 0;
      }
    }
    __syncthreads();
  }
}

// Far signs of the result of a pointwise boolean for unallocated bricks.
template <class T, class Comp>
__global__ void kPointwise2FarSign(int nBricks, const int8_t *fa,
                                   const int8_t *fb, int8_t *fo, Comp comp) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nBricks;
       b += gridDim.x * blockDim.x) {
    bool mv = false;
    const T a = fa[b] < 0 ? Lim<T>::lowest() : Lim<T>::max();
    const T bb = fb[b] < 0 ? Lim<T>::lowest() : Lim<T>::max();
    const T o = comp(a, bb, mv);
    fo[b] = o < 0 ? -1 : 1;
  }
}

template <class T> struct MaxComp { // INTERSECT, lsBooleanOperation.hpp:270-276
  __device__ T operator()(T a, T b, bool &) const { return a > b ? a : b; }
};
template <class T> struct MinComp { // UNION, :262-268
  __device__ T operator()(T a, T b, bool &) const { return a < b ? a : b; }
};
template <class T> struct RelComplementComp { // :278-280
  __device__ T operator()(T a, T b, bool &) const { return a > -b ? a : -b; }
};
// combineLevelSets comparator, lsAdvect.hpp:218-230 (a = current, b = saved).
// The stage combination is evaluated in double for both storage types: for
// T = double this is the reference's expression, for T = float it is the
// precision form's FP64 stage combination, rounded once to float.
template <class T> struct CombineComp {
  double wTarget, wSource;
  __device__ T operator()(T a, T b, bool &moved) const {
    if (isDef(a) && isDef(b)) {
      const T res = T(wSource * (double)a + wTarget * (double)b);
      if (res > b) moved = true;
      return res;
    }
    if (!isDef(a)) return a;
    return b;
  }
};

} // namespace vlsg
