// vlso_core.hpp -- TEST INFRASTRUCTURE ONLY (the oracle): an FP64 C++/OpenMP
// restatement of the band-maintenance rules of ViennaLS 5.8.3 that
// viennals::Advect<double,D>::apply runs.  It is the checker for the CUDA
// library and the CPU baseline; nothing in the product links it.
//
// Parity status: the rules below are restated from the reference headers
// (file:line cited per function).  ViennaHRLE 1.1.2, which stores the
// reference's level sets, is not available, so its iteration semantics are
// restated too: x fastest / highest dimension slowest order, undefined points
// read as +-numeric_limits<double>::max() carrying their run's sign, the
// periodic wrap (points min..max-1) and the reflective mirror (2*min-i,
// 2*max-i) -- the last two are NOT pinned against a real HRLE build.
//
// Representation: a level set is a sorted map key -> value holding every
// defined point plus every undefined star-neighbour of a defined point (the
// "shell"), the latter with its sentinel (+-max).  Every rule of the
// reference maps an undefined point whose star-neighbourhood is undefined to
// an undefined point of the same sign, so only map points can change in a
// pass; the sign of a point outside the map is found by walking through
// undefined points to the nearest map point (undefined neighbours of a valid
// level set share their sign, lsCheck.hpp:125-138).
#pragma once

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include <omp.h>

#include "../include/vlsg.h"

namespace vlso {

constexpr double POS = std::numeric_limits<double>::max();     // lsDomain.hpp:51
constexpr double NEG = std::numeric_limits<double>::lowest();  // lsDomain.hpp:52
constexpr double EPS = std::numeric_limits<double>::epsilon();

inline bool isDefined(double v) { return v != POS && v != NEG; }
inline double undefinedOf(double v) { return v < 0 ? NEG : POS; }

// 21 bits per coordinate, offset 2^20; x in the low bits so that sorting keys
// sorts in HRLE order (x fastest, highest dimension slowest).
constexpr int KB = 21;
constexpr int64_t KOFF = int64_t(1) << 20;
constexpr uint64_t KMASK = (uint64_t(1) << KB) - 1;

template <int D> struct Grid {
  int64_t minI[D], maxI[D];
  int bc[D];
  double delta;

  // Index mapping of one coordinate through the boundary condition.
  int64_t mapCoord(int d, int64_t c) const {
    switch (bc[d]) {
    case VLSG_PERIODIC_BOUNDARY: {
      const int64_t n = maxI[d] - minI[d];
      if (n <= 0) return minI[d];
      int64_t r = (c - minI[d]) % n;
      if (r < 0) r += n;
      return minI[d] + r;
    }
    case VLSG_REFLECTIVE_BOUNDARY: {
      if (maxI[d] <= minI[d]) return minI[d];
      for (int guard = 0; guard < 64; ++guard) {
        if (c < minI[d]) c = 2 * minI[d] - c;
        else if (c > maxI[d]) c = 2 * maxI[d] - c;
        else break;
      }
      return c;
    }
    case VLSG_POS_INFINITE_BOUNDARY:
      return c < minI[d] ? 2 * minI[d] - c : c;
    case VLSG_NEG_INFINITE_BOUNDARY:
      return c > maxI[d] ? 2 * maxI[d] - c : c;
    default:
      return c;
    }
  }
  bool bounded(int d) const {
    return bc[d] == VLSG_PERIODIC_BOUNDARY || bc[d] == VLSG_REFLECTIVE_BOUNDARY;
  }
  // number of distinct points along a bounded direction
  int64_t extent(int d) const {
    return bc[d] == VLSG_PERIODIC_BOUNDARY ? maxI[d] - minI[d]
                                           : maxI[d] - minI[d] + 1;
  }
};

template <int D> inline uint64_t encode(const int64_t *c) {
  uint64_t k = 0;
  for (int d = D - 1; d >= 0; --d) k = (k << KB) | uint64_t(c[d] + KOFF);
  return k;
}
template <int D> inline void decode(uint64_t k, int64_t *c) {
  for (int d = 0; d < D; ++d) {
    c[d] = int64_t(k & KMASK) - KOFF;
    k >>= KB;
  }
}
template <int D> inline int64_t coordOf(uint64_t k, int d) {
  return int64_t((k >> (KB * d)) & KMASK) - KOFF;
}
template <int D> inline uint64_t withCoord(uint64_t k, int d, int64_t c) {
  const uint64_t m = KMASK << (KB * d);
  return (k & ~m) | (uint64_t(c + KOFF) << (KB * d));
}
// key of the point `off` away along direction d, mapped through the BC
template <int D>
inline uint64_t shiftKey(const Grid<D> &g, uint64_t k, int d, int64_t off) {
  return withCoord<D>(k, d, g.mapCoord(d, coordOf<D>(k, d) + off));
}
template <int D>
inline uint64_t offsetKey(const Grid<D> &g, uint64_t k, const int *off) {
  for (int d = 0; d < D; ++d)
    if (off[d]) k = shiftKey<D>(g, k, d, off[d]);
  return k;
}

// Open-addressing index key -> position, built in parallel.
struct HashIndex {
  std::vector<std::atomic<uint64_t>> slots;
  std::vector<int64_t> pos;
  uint64_t mask = 0;
  int shift = 64;
  static constexpr uint64_t EMPTY = ~uint64_t(0);

  void build(const std::vector<uint64_t> &keys) {
    uint64_t cap = 16;
    int bits = 4;
    while (cap < 2 * keys.size() + 16) cap <<= 1, ++bits;
    std::vector<std::atomic<uint64_t>> s(cap);
    slots.swap(s);
    pos.assign(cap, -1);
    mask = cap - 1;
    shift = 64 - bits;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)cap; ++i)
      slots[i].store(EMPTY, std::memory_order_relaxed);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)keys.size(); ++i) {
      uint64_t h = (keys[i] * 0x9E3779B97F4A7C15ull) >> shift;
      for (;;) {
        uint64_t expect = EMPTY;
        if (slots[h].compare_exchange_strong(expect, keys[i])) {
          pos[h] = i;
          break;
        }
        h = (h + 1) & mask;
      }
    }
  }
  int64_t find(uint64_t k) const {
    if (slots.empty()) return -1;
    uint64_t h = (k * 0x9E3779B97F4A7C15ull) >> shift;
    for (;;) {
      const uint64_t s = slots[h].load(std::memory_order_relaxed);
      if (s == k) return pos[h];
      if (s == EMPTY) return -1;
      h = (h + 1) & mask;
    }
  }
};

// Point data of one defined point while it is carried through the passes
// (translateFromMultiData with the source point ids the reference's Expand,
// Reduce, Prune, BooleanOperation and rebuildLS record: lsExpand.hpp:110-150,
// lsReduce.hpp:108-112, lsPrune.hpp:164-168, lsBooleanOperation.hpp:104-114,
// lsAdvect.hpp:318-410): the index of the point, at the start of the
// advection, whose data it carries (-1: none), and the AdvectionVelocities /
// Dissipation values of the last value update (lsAdvect.hpp:780-796).
struct PointData {
  int64_t src = -1;
  double vel = 0., diss = 0.;
};

template <int D> struct LS {
  Grid<D> grid;
  std::vector<uint64_t> keys; // sorted, HRLE order
  std::vector<double> vals;   // defined value or +-max (shell)
  int width = 1;              // Domain::levelSetWidth, lsDomain.hpp:42
  double emptyValue = POS;    // the value everywhere when the map is empty
  HashIndex index;
  int64_t nDefined = 0;
  mutable std::atomic<int64_t> farQueries{0};
  // point data per map entry (empty: not tracked)
  std::vector<PointData> pd;

  LS() = default;
  LS(const LS &o)
      : grid(o.grid), keys(o.keys), vals(o.vals), width(o.width), emptyValue(o.emptyValue),
        nDefined(o.nDefined), pd(o.pd) {
    index.build(keys);
  }
  LS &operator=(const LS &o) {
    grid = o.grid;
    keys = o.keys;
    vals = o.vals;
    width = o.width;
    emptyValue = o.emptyValue;
    nDefined = o.nDefined;
    pd = o.pd;
    index.build(keys);
    return *this;
  }
  void finalizeMap() {
    index.build(keys);
    int64_t n = 0;
#pragma omp parallel for reduction(+ : n)
    for (int64_t i = 0; i < (int64_t)vals.size(); ++i)
      n += isDefined(vals[i]) ? 1 : 0;
    nDefined = n;
  }

  // Value of any grid point: map value, or the sign of the undefined region
  // it lies in.
  double at(uint64_t k) const {
    const int64_t p = index.find(k);
    if (p >= 0) return vals[p];
    return farValue(k);
  }

  // Sign of an undefined point outside the map: walk along x (sorted rows),
  // then along the other axes, to the first map point; fall back to the
  // L1-nearest map point.  An empty level set is positive everywhere
  // (a new Domain is filled with POS_VALUE, lsDomain.hpp:64-65).
  double farValue(uint64_t k) const {
    farQueries.fetch_add(1, std::memory_order_relaxed);
    if (keys.empty()) return emptyValue;
    // 1. same x-row (keys of a row are contiguous)
    const uint64_t row = k >> KB;
    auto it = std::lower_bound(keys.begin(), keys.end(), k);
    int64_t best = -1, bestDist = INT64_MAX;
    if (it != keys.end() && ((*it) >> KB) == row) {
      best = it - keys.begin();
      bestDist = int64_t(*it - k);
    }
    if (it != keys.begin() && ((*(it - 1)) >> KB) == row) {
      const int64_t d = int64_t(k - *(it - 1));
      if (d < bestDist) best = (it - 1) - keys.begin(), bestDist = d;
    }
    if (best >= 0) return undefinedOf(vals[best]);
    // 2. along the remaining axes
    for (int d = 1; d < D; ++d) {
      const int64_t lim = grid.bounded(d) ? grid.extent(d) : 4096;
      const int64_t c0 = coordOf<D>(k, d);
      for (int64_t t = 1; t <= lim; ++t) {
        for (int s = -1; s <= 1; s += 2) {
          const uint64_t kk = withCoord<D>(k, d, grid.mapCoord(d, c0 + s * t));
          const int64_t p = index.find(kk);
          if (p >= 0) return undefinedOf(vals[p]);
        }
      }
    }
    // 3. L1-nearest map point
    int64_t c[D];
    decode<D>(k, c);
    int64_t bi = 0, bd = INT64_MAX;
    for (int64_t i = 0; i < (int64_t)keys.size(); ++i) {
      int64_t q[D];
      decode<D>(keys[i], q);
      int64_t dist = 0;
      for (int d = 0; d < D; ++d) dist += std::llabs(q[d] - c[d]);
      if (dist < bd) bd = dist, bi = i;
    }
    return undefinedOf(vals[bi]);
  }
};

// ---------------------------------------------------------------------------
// Building a map from defined points and run signs

// Sign of an undefined point from the HRLE run list: the last undefined run
// starting at or before the point (runs and defined points tile the order).
struct RunSigns {
  std::vector<uint64_t> start;
  std::vector<int8_t> sign;
  double at(uint64_t k) const {
    if (start.empty()) return POS;
    auto it = std::upper_bound(start.begin(), start.end(), k);
    if (it == start.begin()) return sign[0] < 0 ? NEG : POS;
    return sign[(it - start.begin()) - 1] < 0 ? NEG : POS;
  }
};

// Collect (defined points) + (star shell) into a fresh sorted map.  `shellVal`
// gives the value of a shell point, given the key of the shell point and the
// index (into defKeys) of the defined point it was reached from.
// With `defPd` (point data of the defined points) the map carries point data.
template <int D, class ShellFn>
void assembleMap(LS<D> &out, const std::vector<uint64_t> &defKeys,
                 const std::vector<double> &defVals, ShellFn shellVal,
                 const std::vector<PointData> *defPd = nullptr) {
  struct Entry {
    uint64_t key;
    double val;
    int64_t def; // index into defKeys, -1 for a shell point
  };
  const int64_t n = defKeys.size();
  const int nt = omp_get_max_threads();
  std::vector<std::vector<Entry>> shell(nt);
#pragma omp parallel
  {
    auto &loc = shell[omp_get_thread_num()];
#pragma omp for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
      for (int d = 0; d < D; ++d)
        for (int s = -1; s <= 1; s += 2) {
          const uint64_t nk = shiftKey<D>(out.grid, defKeys[i], d, s);
          if (std::binary_search(defKeys.begin(), defKeys.end(), nk)) continue;
          loc.push_back({nk, shellVal(nk, i), -1});
        }
    }
  }
  std::vector<Entry> all;
  all.reserve(n + n);
  for (int64_t i = 0; i < n; ++i) all.push_back({defKeys[i], defVals[i], i});
  for (auto &v : shell) all.insert(all.end(), v.begin(), v.end());
  std::sort(all.begin(), all.end(), [](const Entry &a, const Entry &b) { return a.key < b.key; });
  out.keys.clear();
  out.vals.clear();
  out.pd.clear();
  out.keys.reserve(all.size());
  out.vals.reserve(all.size());
  std::vector<int64_t> from;
  from.reserve(all.size());
  for (size_t i = 0; i < all.size(); ++i) {
    if (i > 0 && all[i].key == all[i - 1].key) {
      // a defined point always wins over a shell copy of itself
      if (isDefined(all[i].val) && !isDefined(out.vals.back())) {
        out.vals.back() = all[i].val;
        from.back() = all[i].def;
      }
      continue;
    }
    out.keys.push_back(all[i].key);
    out.vals.push_back(all[i].val);
    from.push_back(all[i].def);
  }
  if (defPd) {
    out.pd.assign(out.keys.size(), PointData{});
    for (size_t i = 0; i < out.keys.size(); ++i)
      if (from[i] >= 0) out.pd[i] = (*defPd)[from[i]];
  }
  out.finalizeMap();
}

template <int D>
void fromPoints(LS<D> &ls, const Grid<D> &g, int64_t n, const int32_t *idx,
                const double *vals, int64_t nRuns, const int32_t *runStart,
                const int8_t *runSign, int width) {
  ls.grid = g;
  ls.width = width;
  std::vector<std::pair<uint64_t, double>> pts(n);
  for (int64_t i = 0; i < n; ++i) {
    int64_t c[D];
    for (int d = 0; d < D; ++d) c[d] = g.mapCoord(d, idx[i * D + d]);
    pts[i] = {encode<D>(c), vals[i]};
  }
  std::sort(pts.begin(), pts.end());
  std::vector<uint64_t> k;
  std::vector<double> v;
  for (auto &p : pts) {
    if (!k.empty() && k.back() == p.first)
      throw std::runtime_error("duplicate defined point");
    if (!isDefined(p.second)) continue;
    k.push_back(p.first);
    v.push_back(p.second);
  }
  RunSigns rs;
  std::vector<std::pair<uint64_t, int8_t>> runs(nRuns);
  for (int64_t i = 0; i < nRuns; ++i) {
    int64_t c[D];
    for (int d = 0; d < D; ++d) c[d] = runStart[i * D + d];
    runs[i] = {encode<D>(c), runSign[i]};
  }
  std::sort(runs.begin(), runs.end());
  for (auto &r : runs) rs.start.push_back(r.first), rs.sign.push_back(r.second);
  assembleMap<D>(ls, k, v, [&](uint64_t nk, int64_t) { return rs.at(nk); });
}

// Generic star pass over all map points.  `rule(centerValue, nb[2D])`
// returns the new value of a point from itself and its 2D star neighbours,
// neighbour order +e_0..+e_{D-1}, -e_0..-e_{D-1} as the reference's
// ConstSparseStarIterator<.,1> numbers them (lsWENO.hpp:252-256).  Every rule
// used with it maps an all-undefined neighbourhood to the centre's own
// undefined value, which makes points outside the map invariant.
// `rule(center, nb, src)` also names the point whose data the result
// carries: src = -1 the centre, 0..2D-1 neighbour src, -2 none.
template <int D, class Rule> void starPass(LS<D> &ls, Rule rule) {
  const int64_t n = ls.keys.size();
  std::vector<double> out(n);
  std::vector<int> srcOf(n, -1);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    double nb[2 * D];
    for (int d = 0; d < D; ++d) {
      for (int s = 0; s < 2; ++s) {
        const uint64_t nk = shiftKey<D>(ls.grid, ls.keys[i], d, s ? -1 : 1);
        const int64_t p = ls.index.find(nk);
        double v;
        if (p >= 0) v = ls.vals[p];
        else if (!isDefined(ls.vals[i])) v = ls.vals[i];
        else v = ls.farValue(nk);
        nb[s * D + d] = v;
      }
    }
    out[i] = rule(ls.vals[i], nb, srcOf[i]);
  }
  std::vector<uint64_t> dk;
  std::vector<double> dv;
  std::vector<int64_t> from;
  for (int64_t i = 0; i < n; ++i)
    if (isDefined(out[i])) dk.push_back(ls.keys[i]), dv.push_back(out[i]), from.push_back(i);
  std::vector<PointData> dpd;
  const bool track = !ls.pd.empty();
  if (track) {
    dpd.resize(dk.size());
    for (size_t j = 0; j < dk.size(); ++j) {
      const int64_t i = from[j];
      const int src = srcOf[i];
      if (src == -1) {
        dpd[j] = ls.pd[i];
      } else if (src >= 0) {
        const int d = src % D, sgn = src < D ? 1 : -1;
        const int64_t p = ls.index.find(shiftKey<D>(ls.grid, ls.keys[i], d, sgn));
        dpd[j] = p >= 0 ? ls.pd[p] : PointData{};
      }
    }
  }
  LS<D> res;
  res.grid = ls.grid;
  res.width = ls.width;
  assembleMap<D>(res, dk, dv, [&](uint64_t nk, int64_t j) {
    const int64_t p = ls.index.find(nk);
    if (p >= 0) return out[p]; // undefined here: defined ones come from dk
    // not in the old map: unchanged undefined point; its sign is that of the
    // (then undefined) point it is adjacent to
    const double old = ls.vals[from[j]];
    return isDefined(old) ? ls.farValue(nk) : old;
  }, track ? &dpd : nullptr);
  ls.keys.swap(res.keys);
  ls.vals.swap(res.vals);
  ls.pd.swap(res.pd);
  ls.finalizeMap();
}

// Expand::apply, lsExpand.hpp:44-172.
template <int D> void expand(LS<D> &ls, int width) {
  if (width <= ls.width) return;        // :52-53
  if (ls.nDefined == 0) return;         // :55-56
  const double totalLimit = width * 0.5; // :58
  const int startWidth = ls.width;
  const int cycles = width - startWidth;
  for (int c = 0; c < cycles; ++c) {
    const double limit = (startWidth + c + 1) * double(0.5); // :67
    starPass<D>(ls, [&](double center, const double *nb, int &src) {
      if (std::abs(center) <= totalLimit) return center; // :108-112
      if (center > -EPS) {                                // :114
        double distance = POS;
        for (int i = 0; i < 2 * D; ++i) {
          const double nv = nb[i] + double(1);
          if (distance > nv) distance = nv, src = i;
        }
        return distance <= limit ? distance : POS; // :124-134
      }
      double distance = NEG;
      for (int i = 0; i < 2 * D; ++i) {
        const double nv = nb[i] - double(1);
        if (distance < nv) distance = nv, src = i;
      }
      return distance >= -limit ? distance : NEG; // :145-155
    });
  }
  ls.width = width; // :171
}

// Reduce::apply, lsReduce.hpp:55-134 (pointwise; the shell of the result is
// rebuilt from the reduced defined set).
template <int D> void reduce(LS<D> &ls, int width) {
  if (width >= ls.width) return; // :241-242
  const double valueLimit = width * 0.5;
  std::vector<uint64_t> dk;
  std::vector<double> dv;
  std::vector<PointData> dpd;
  std::vector<double> newVal(ls.vals.size());
  const bool track = !ls.pd.empty();
  for (size_t i = 0; i < ls.vals.size(); ++i) {
    const double v = ls.vals[i];
    if (isDefined(v) && std::abs(v) <= valueLimit) {
      dk.push_back(ls.keys[i]);
      dv.push_back(v);
      if (track) dpd.push_back(ls.pd[i]);
      newVal[i] = v;
    } else {
      newVal[i] = v < 0 ? NEG : POS; // :292-295
    }
  }
  LS<D> res;
  res.grid = ls.grid;
  assembleMap<D>(res, dk, dv, [&](uint64_t nk, int64_t) {
    const int64_t p = ls.index.find(nk);
    return p >= 0 ? newVal[p] : ls.farValue(nk);
  }, track ? &dpd : nullptr);
  ls.keys.swap(res.keys);
  ls.vals.swap(res.vals);
  ls.pd.swap(res.pd);
  ls.finalizeMap();
  ls.width = width; // :311
}

// Prune::apply, lsPrune.hpp:74-195.
template <int D> void prune(LS<D> &ls, bool removeStrayZeros) {
  if (ls.nDefined == 0) return; // :81-83
  auto isNegative = [](double a) { return a <= -EPS; };                 // :22-24
  auto isSignDifferent = [&](double a, double b) -> bool {              // :26-29
    return isNegative(a) != isNegative(b);
  };
  auto isSignDifferentOrZero = [&](double a, double b) -> bool {                // :31-36
    if (a == 0. || b == 0.) return true;
    return isSignDifferent(a, b);
  };
  auto isMonotone = [&](double a, double c) -> bool {                           // :50-52
    return a == 0. || c == 0. || isSignDifferent(a, c);
  };
  starPass<D>(ls, [&](double center, const double *nb, int &src) {
    const bool centerSign = isNegative(center);
    if (!isDefined(center)) return centerSign ? NEG : POS; // :175-179
    bool keepPoint = true;
    if (std::abs(center) != 0.) {                           // :126
      keepPoint = false;
      for (int i = 0; i < 2 * D; ++i) {
        const bool diff = removeStrayZeros ? isSignDifferentOrZero(center, nb[i])
                                           : isSignDifferent(center, nb[i]);
        if (diff) { keepPoint = true; break; }
      }
    }
    if (removeStrayZeros && std::abs(center) == 0.) {       // :135-160
      for (int i = 0; i < D; ++i) {
        const double negVal = nb[i];     // getNeighbor(i)   = +e_i
        const double posVal = nb[D + i]; // getNeighbor(D+i) = -e_i
        // the reference records no source for this point (lsPrune.hpp:
        // 150-155 inserts it without a data id)
        if (!isMonotone(negVal, posVal)) {
          src = -2;
          return std::abs(negVal) < std::abs(posVal) ? negVal : posVal;
        }
      }
    }
    if (keepPoint) return center;
    return centerSign ? NEG : POS; // :168-174
  });
  ls.width = 2; // :193
}

// BooleanOperation::booleanOpInternal, lsBooleanOperation.hpp:59-213, with
// the comparator over (A value, B value) -> (value, fromA).  Points of A's
// and B's maps are visited; everything else is undefined in both and the
// comparator of two sentinels is again a sentinel.
// `fromA(a, b)`: whether a defined result takes A's point data (the
// comparator's second value); results from B take B's, or none when B
// carries no point data (lsBooleanOperation.hpp:160-196).
inline bool neverFromA(double, double) { return false; }
template <int D, class Comp, class FromA = bool (*)(double, double)>
void booleanOp(LS<D> &A, const LS<D> &B, Comp comp, bool pruneResult = true,
               FromA fromA = neverFromA) {
  std::vector<uint64_t> cand;
  cand.reserve(A.keys.size() + B.keys.size());
  std::merge(A.keys.begin(), A.keys.end(), B.keys.begin(), B.keys.end(),
             std::back_inserter(cand));
  cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
  const int64_t n = cand.size();
  std::vector<double> out(n), va(n), vb(n);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    va[i] = A.at(cand[i]);
    vb[i] = B.at(cand[i]);
    out[i] = comp(va[i], vb[i]);
  }
  std::vector<uint64_t> dk;
  std::vector<double> dv;
  std::vector<int64_t> from;
  for (int64_t i = 0; i < n; ++i)
    if (isDefined(out[i])) dk.push_back(cand[i]), dv.push_back(out[i]), from.push_back(i);
  const bool track = !A.pd.empty();
  std::vector<PointData> dpd;
  if (track) {
    dpd.resize(dk.size());
    for (size_t j = 0; j < dk.size(); ++j) {
      const int64_t i = from[j];
      if (fromA(va[i], vb[i])) {
        const int64_t p = A.index.find(cand[i]);
        if (p >= 0) dpd[j] = A.pd[p];
      } else if (!B.pd.empty()) {
        const int64_t p = B.index.find(cand[i]);
        if (p >= 0) dpd[j] = B.pd[p];
      }
    }
  }
  LS<D> res;
  res.grid = A.grid;
  assembleMap<D>(res, dk, dv, [&](uint64_t nk, int64_t j) {
    auto it = std::lower_bound(cand.begin(), cand.end(), nk);
    if (it != cand.end() && *it == nk) {
      const double o = out[it - cand.begin()];
      return isDefined(o) ? undefinedOf(o) : o; // defined ones come from dk
    }
    const int64_t f = from[j];
    const double a = isDefined(va[f]) ? A.farValue(nk) : va[f];
    const double b = isDefined(vb[f]) ? B.farValue(nk) : vb[f];
    return comp(a, b);
  }, track ? &dpd : nullptr);
  const int widthA = A.width;
  A.keys.swap(res.keys);
  A.vals.swap(res.vals);
  A.pd.swap(res.pd);
  A.finalizeMap();
  A.width = widthA; // :201
  if (pruneResult) { // :203-210
    prune<D>(A, true);
    prune<D>(A, false);
  }
}

inline double minComp(double a, double b) { return a < b ? a : b; } // :262-268
inline double maxComp(double a, double b) { return a > b ? a : b; } // :270-276
inline bool minFromA(double a, double b) { return a < b; }
inline bool maxFromA(double a, double b) { return a > b; }

// lsAdvect.hpp:238-429, rebuildLS.
// With updateData false the new level set carries no point data
// (lsAdvect.hpp:418-423 translates it only when updatePointData is set).
template <int D>
void rebuild(LS<D> &ls, double cutoff, int finalWidth, bool updateData = true) {
  starPass<D>(ls, [&](double c, const double *nb, int &src) {
    if (std::abs(c) <= 1.0) { // :306
      int k = 0;
      for (; k < 2 * D; k++)
        if (std::signbit(nb[k] - 1e-7) != std::signbit(c + 1e-7)) break;
      if (k != 2 * D) {
        if (c > 0.5) {
          int j = 0;
          for (; j < 2 * D; j++)
            if (std::abs(nb[j]) <= 1.0)
              if (nb[j] < -0.5) break;
          if (j != 2 * D) src = j;
          return j == 2 * D ? c : 0.5;
        } else if (c < -0.5) {
          int j = 0;
          for (; j < 2 * D; j++)
            if (std::abs(nb[j]) <= 1.0)
              if (nb[j] > 0.5) break;
          if (j != 2 * D) src = j;
          return j == 2 * D ? c : -0.5;
        }
        return c;
      }
      return c < 0 ? NEG : POS; // :359-364
    }
    if (c >= 0) { // :367
      double distance = POS;
      for (int i = 0; i < 2 * D; i++) {
        const double value = nb[i];
        if (std::abs(value) <= 1.0 && (value < 0.))
          if (distance > value + 1.0) distance = value + 1.0, src = i;
      }
      return distance <= cutoff ? distance : POS;
    }
    double distance = NEG;
    for (int i = 0; i < 2 * D; i++) {
      const double value = nb[i];
      if (std::abs(value) <= 1.0 && (value > 0))
        if (distance < value - 1.0) distance = value - 1.0, src = i;
    }
    return distance >= -cutoff ? distance : NEG;
  });
  if (!updateData) ls.pd.clear();
  ls.width = finalWidth; // :428
}

// BooleanOperation INVERT, lsBooleanOperation.hpp:215-255: every value
// negated, undefined signs swapped; the width is kept.
template <int D> void invert(LS<D> &ls) {
  for (auto &v : ls.vals) v = -v;
  ls.emptyValue = -ls.emptyValue;
  ls.finalizeMap();
}

// PrepareStencilLocalLaxFriedrichs, lsStencilLocalLaxFriedrichsScalar.hpp:
// 423-477.  The reference tests a layer with isDepo[isDepo[i]] (:448: it
// indexes the vector with the element); kept, with an index past the end
// read as false.
template <int D> void prepareStencilLLF(std::vector<LS<D>> &lss, std::vector<bool> isDepo) {
  const int L = (int)lss.size();
  isDepo.resize(L, false);
  LS<D> finalTop;
  finalTop.grid = lss[0].grid;
  finalTop.width = 1;
  finalTop.finalizeMap();
  auto relComp = [](double a, double b) { return maxComp(a, -b); };
  bool layerAboveIsDepo = false;
  int layer = L - 1;
  for (int i = L - 1; i >= 0; --i) {
    const size_t e = isDepo[i] ? 1 : 0;
    const bool depo = e < isDepo.size() && isDepo[e];
    if (depo) {
      if (!layerAboveIsDepo) {
        layer = i;
        layerAboveIsDepo = true;
      }
    } else {
      if (layerAboveIsDepo) {
        LS<D> layerAbove = lss[layer];
        booleanOp<D>(layerAbove, lss[i], relComp);
        booleanOp<D>(finalTop, layerAbove, minComp);
        prune<D>(finalTop, false);
      }
      layerAboveIsDepo = false;
    }
  }
  if (layerAboveIsDepo) booleanOp<D>(finalTop, lss[layer], minComp);
  invert<D>(finalTop);
  lss.back() = finalTop;
}

// FinalizeStencilLocalLaxFriedrichs, :480-492.
template <int D> void finalizeStencilLLF(std::vector<LS<D>> &lss) {
  LS<D> &top = lss.back();
  invert<D>(top);
  booleanOp<D>(top, lss[lss.size() - 2], minComp);
}

} // namespace vlso
