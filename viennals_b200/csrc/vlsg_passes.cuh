// vlsg_passes.cuh -- the rules of the band passes of libvlsgpu.
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
// The kernels that apply them are in vlsg_frontier.cuh.
#pragma once

#include "vlsg_common.cuh"

namespace vlsg {
namespace { // internal linkage: every compilation unit has its own copy

// Every rule also names the cell whose point data its result carries (the
// source ids of the reference's passes): src -1 the centre, 0..5 star
// neighbour src, -2 none.
// Sign classes are decided with the FP64 epsilon in both precisions: the FP32
// precision form follows the decisions of Advect<double>, the path it is held
// to (Advect<float> would compare with FLT_EPSILON).
template <class T> struct ExpandRule {
  T totalLimit, limit;
  __device__ T operator()(T c, const T *nb, int &src) const {
    if (fabs(c) <= totalLimit) return c;
    if ((double)c > -Lim<double>::eps()) {
      T distance = Lim<T>::max();
      for (int i = 0; i < 6; ++i) {
        const T nv = nb[i] + T(1);
        if (distance > nv) distance = nv, src = i;
      }
      return distance <= limit ? distance : Lim<T>::max();
    }
    T distance = Lim<T>::lowest();
    for (int i = 0; i < 6; ++i) {
      const T nv = nb[i] - T(1);
      if (distance < nv) distance = nv, src = i;
    }
    return distance >= -limit ? distance : Lim<T>::lowest();
  }
};

// Expand of a D = 2 level set held as the plane of a z-periodic grid of
// period 1 (GridDev::planar): the z neighbours (2, 5) are the cell itself,
// which the 2D star does not have; they read as undefined on the side the
// rule takes for the cell, which never decides the result (a defined cell
// recomputed from its neighbours would otherwise see its own value +-1).
// Prune and rebuild need no such rule: a cell's own sign class and value
// never decide them.
template <class T> struct PlanarExpandRule {
  ExpandRule<T> r;
  __device__ T operator()(T c, const T *nb, int &src) const {
    const T self = (double)c > -Lim<double>::eps() ? Lim<T>::max() : Lim<T>::lowest();
    const T nb4[6] = {nb[0], nb[1], self, nb[3], nb[4], self};
    return r(c, nb4, src);
  }
};

template <class T> struct PruneRule {
  bool removeStrayZeros;
  __device__ static bool neg(T a) { return (double)a <= -Lim<double>::eps(); }
  __device__ static bool diff(T a, T b) { return neg(a) != neg(b); }
  __device__ T operator()(T c, const T *nb, int &src) const {
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
        // inserted without a data id by the reference (lsPrune.hpp:150-155)
        if (!monotone) {
          src = -2;
          return fabs(a) < fabs(b) ? a : b;
        }
      }
    }
    if (keep) return c;
    return cneg ? Lim<T>::lowest() : Lim<T>::max();
  }
};

template <class T> struct RebuildRule {
  double cutoff;
  __device__ T operator()(T cT, const T *nb, int &src) const {
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
          if (j != 6) src = j;
          return j == 6 ? cT : T(0.5);
        } else if (c < -0.5) {
          int j = 0;
          for (; j < 6; j++)
            if (fabs((double)nb[j]) <= 1.0 && (double)nb[j] > 0.5) break;
          if (j != 6) src = j;
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
          if ((double)distance > v + 1.0) distance = T(v + 1.0), src = i;
      }
      return (double)distance <= cutoff ? distance : Lim<T>::max();
    }
    T distance = Lim<T>::lowest();
    for (int i = 0; i < 6; i++) {
      const double v = (double)nb[i];
      if (fabs(v) <= 1.0 && (v > 0))
        if ((double)distance < v - 1.0) distance = T(v - 1.0), src = i;
    }
    return (double)distance >= -cutoff ? distance : Lim<T>::lowest();
  }
};

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
  static constexpr bool keepsUndefinedA = false;
  __device__ T operator()(T a, T b, bool &) const { return a > b ? a : b; }
};
template <class T> struct MinComp { // UNION, :262-268
  static constexpr bool keepsUndefinedA = false;
  __device__ T operator()(T a, T b, bool &) const { return a < b ? a : b; }
};
template <class T> struct RelComplementComp { // :278-280
  static constexpr bool keepsUndefinedA = false;
  __device__ T operator()(T a, T b, bool &) const { return a > -b ? a : -b; }
};
// combineLevelSets comparator, lsAdvect.hpp:218-230 (a = current, b = saved).
// The stage combination is evaluated in double for both storage types: for
// T = double this is the reference's expression, for T = float it is the
// precision form's FP64 stage combination, rounded once to float.
template <class T> struct CombineComp {
  // an undefined current value stays as it is: only defined cells can change
  static constexpr bool keepsUndefinedA = true;
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
  // both defined, as hi + lo sums in double (FP32 buffers with compensation
  // terms): the stage combination without rounding to the storage type
  __device__ double full(double a, double b, bool &moved) const {
    const double res = wSource * a + wTarget * b;
    if (res > b) moved = true;
    return res;
  }
};

} // namespace
} // namespace vlsg
