// vlso_metrics.hpp -- TEST INFRASTRUCTURE ONLY (the oracle): validity check
// (lsCheck.hpp:51-155) and the Chamfer comparison (lsCompareChamfer.hpp:104-
// 242) on the zero-crossing nodes that lsToSurfaceMesh.hpp:102-412 places on
// grid edges (sharp corners off, the default).  Node merging follows
// insertNode (0.05-grid-unit bins, position averaging); nodes are visited in
// HRLE order of their edge's lower end point, an approximation of the
// marching-cubes triangle order that only changes which merged node a bin
// keeps.
#pragma once

#include <unordered_map>

#include "vlso_core.hpp"

namespace vlso {

// Check::GetStatusFromDistance, lsCheck.hpp:51-58
inline int statusFromDistance(double value) {
  int x = static_cast<int>(value);
  if (value >= 0.) return (value <= double(x) + 0.5) ? x : x + 1;
  return (value >= double(x) - 0.5) ? x : x - 1;
}

// Check::apply, lsCheck.hpp:78-155; returns the number of faults.
template <int D> int64_t check(const LS<D> &ls) {
  auto isNegative = [](double v) { return v <= -EPS; };
  int64_t faults = 0;
#pragma omp parallel for reduction(+ : faults) schedule(static)
  for (int64_t p = 0; p < (int64_t)ls.keys.size(); ++p) {
    const double c = ls.vals[p];
    for (int d = 0; d < D; ++d)
      for (int s = -1; s <= 1; s += 2) {
        const uint64_t nk = shiftKey<D>(ls.grid, ls.keys[p], d, s);
        const double n = ls.at(nk);
        if (isDefined(c)) {
          if (isDefined(n)) {
            if (std::abs(statusFromDistance(c) - statusFromDistance(n)) > 1)
              ++faults;
          } else if (n >= 0.) {
            if (c < -0.5) ++faults;
          } else {
            if (c > 0.5) ++faults;
          }
        } else if (!isDefined(n)) {
          if (isNegative(c) != isNegative(n)) ++faults;
        }
      }
  }
  return faults;
}

// Zero-crossing nodes on grid edges (physical coordinates, D values each).
template <int D>
std::vector<double> surfaceNodes(const LS<D> &ls, double minNodeDistance = 0.05,
                                 double epsilon = 1e-12) {
  struct Edge {
    uint64_t key;
    int dir;
    double pos[3];
  };
  const int nt = omp_get_max_threads();
  std::vector<std::vector<Edge>> loc(nt);
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < (int64_t)ls.keys.size(); ++p) {
    const double d0 = ls.vals[p];
    if (!isDefined(d0)) continue;
    int64_t c[D];
    decode<D>(ls.keys[p], c);
    for (int dir = 0; dir < D; ++dir) {
      // lower end of the edge is this point; the upper one is +e_dir
      const uint64_t qk = shiftKey<D>(ls.grid, ls.keys[p], dir, 1);
      const double d1 = ls.at(qk);
      if (!isDefined(d1)) continue;
      if ((d0 >= 0.) == (d1 >= 0.)) continue;
      Edge e;
      e.key = ls.keys[p];
      e.dir = dir;
      for (int z = 0; z < 3; ++z) e.pos[z] = 0;
      for (int z = 0; z < D; ++z) {
        if (z != dir) {
          e.pos[z] = double(c[z]);
        } else {
          // interpWithOffset, lsToSurfaceMesh.hpp:339-361
          double cc;
          if (d0 == -d1)
            cc = double(c[z]) + 0.5;
          else if (std::abs(d0) <= std::abs(d1))
            cc = double(c[z]) + (d0 / (d0 - d1));
          else
            cc = double(c[z] + 1) - (d1 / (d1 - d0));
          cc = std::max(cc, double(c[z]) + epsilon);
          cc = std::min(cc, double(c[z] + 1) - epsilon);
          e.pos[z] = cc;
        }
      }
      loc[omp_get_thread_num()].push_back(e);
    }
  }
  std::vector<Edge> edges;
  for (auto &v : loc) edges.insert(edges.end(), v.begin(), v.end());
  std::sort(edges.begin(), edges.end(), [](const Edge &a, const Edge &b) {
    return a.key != b.key ? a.key < b.key : a.dir < b.dir;
  });
  // insertNode, lsToSurfaceMesh.hpp (quantised bins, averaging)
  struct BinHash {
    size_t operator()(const std::array<long long, 3> &k) const {
      uint64_t h = uint64_t(k[0]) * 0x9E3779B185EBCA87ull;
      h ^= uint64_t(k[1]) + 0xC2B2AE3D27D4EB4Full + (h << 6) + (h >> 2);
      h ^= uint64_t(k[2]) + 0x165667B19E3779F9ull + (h << 6) + (h >> 2);
      return size_t(h);
    }
  };
  std::unordered_map<std::array<long long, 3>, size_t, BinHash> bins;
  std::vector<std::array<double, 3>> nodes;
  const double inv = 1.0 / minNodeDistance;
  for (auto &e : edges) {
    std::array<double, 3> pos{e.pos[0], e.pos[1], e.pos[2]};
    std::array<long long, 3> q{std::llround(pos[0] * inv),
                               std::llround(pos[1] * inv),
                               std::llround(pos[2] * inv)};
    auto it = bins.find(q);
    if (it != bins.end()) {
      auto &n = nodes[it->second];
      for (int z = 0; z < 3; ++z) n[z] = (n[z] + pos[z]) * 0.5;
      continue;
    }
    bins.emplace(q, nodes.size());
    nodes.push_back(pos);
  }
  std::vector<double> out(nodes.size() * D);
  for (size_t i = 0; i < nodes.size(); ++i)
    for (int z = 0; z < D; ++z) out[i * D + z] = nodes[i][z] * ls.grid.delta;
  return out;
}

// Nearest-neighbour distances of `queries` to `points` via a uniform grid.
template <int D>
std::vector<double> nearestDistances(const std::vector<double> &points,
                                     const std::vector<double> &queries,
                                     double h) {
  const int64_t np = points.size() / D, nq = queries.size() / D;
  std::vector<double> out(nq, std::numeric_limits<double>::infinity());
  if (np == 0) return out;
  auto cellOf = [&](const double *x, int64_t *c) {
    for (int d = 0; d < D; ++d) c[d] = (int64_t)std::floor(x[d] / h);
  };
  std::unordered_map<uint64_t, std::vector<int64_t>> grid;
  for (int64_t i = 0; i < np; ++i) {
    int64_t c[D];
    cellOf(&points[i * D], c);
    grid[encode<D>(c)].push_back(i);
  }
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t q = 0; q < nq; ++q) {
    const double *x = &queries[q * D];
    int64_t c[D];
    cellOf(x, c);
    double best = std::numeric_limits<double>::infinity();
    for (int r = 0; r < 100000; ++r) {
      // visit the shell of Chebyshev radius r
      int64_t o[D];
      for (int d = 0; d < D; ++d) o[d] = -r;
      for (;;) {
        int64_t m = 0;
        for (int d = 0; d < D; ++d) m = std::max<int64_t>(m, std::llabs(o[d]));
        if (m == r) {
          int64_t cc[D];
          for (int d = 0; d < D; ++d) cc[d] = c[d] + o[d];
          auto it = grid.find(encode<D>(cc));
          if (it != grid.end())
            for (int64_t i : it->second) {
              double s = 0;
              for (int d = 0; d < D; ++d) {
                const double t = points[i * D + d] - x[d];
                s += t * t;
              }
              s = std::sqrt(s);
              if (s < best) best = s;
            }
        }
        int d = 0;
        for (; d < D; ++d) {
          if (o[d] < r) { ++o[d]; break; }
          o[d] = -r;
        }
        if (d == D) break;
      }
      if (best <= r * h) break;
    }
    out[q] = best;
  }
  return out;
}

// CompareChamfer::apply, lsCompareChamfer.hpp:104-242.
// out: forward, backward, chamfer, rms, max.
template <int D>
void chamfer(const LS<D> &target, const LS<D> &sample, double *out,
             int64_t *counts) {
  auto expanded = [](const LS<D> &ls) {
    LS<D> w(ls);
    if (w.width < 2) expand<D>(w, 2); // :118-138
    return w;
  };
  const LS<D> t = expanded(target), s = expanded(sample);
  const auto tn = surfaceNodes<D>(t), sn = surfaceNodes<D>(s);
  const int64_t nT = tn.size() / D, nS = sn.size() / D;
  counts[0] = nT;
  counts[1] = nS;
  if (nT == 0 || nS == 0) {
    for (int i = 0; i < 5; ++i) out[i] = std::numeric_limits<double>::infinity();
    return;
  }
  const double h = target.grid.delta;
  const auto fwd = nearestDistances<D>(sn, tn, h);
  const auto bwd = nearestDistances<D>(tn, sn, h);
  double sumF = 0, sqF = 0, maxF = 0, sumB = 0, sqB = 0, maxB = 0;
  for (double d : fwd) sumF += d, sqF += d * d, maxF = std::max(maxF, d);
  for (double d : bwd) sumB += d, sqB += d * d, maxB = std::max(maxB, d);
  out[0] = sumF / nT;
  out[1] = sumB / nS;
  out[2] = (sumF + sumB) / double(nT + nS);
  out[3] = std::sqrt((sqF + sqB) / double(nT + nS));
  out[4] = std::max(maxF, maxB);
}

} // namespace vlso
