// vlsgViennaLS.hpp -- conversions between viennals::Domain<T,D> (D = 2, 3)
// and vlsg::LevelSet, for a ViennaLS build that puts libvlsgpu behind
// viennals::Advect.  Needs the ViennaLS headers (lsDomain.hpp) and
// ViennaHRLE's sparse iterator (hrleSparseIterator.hpp) on the include path.
// Only calls the reference itself makes are used:
//   Grid::getMinIndex / getMaxIndex      lsFromSurfaceMesh.hpp:281-282
//   Grid::getBoundaryConditions          lsExtrude.hpp:34
//   Grid::getGridDelta                   lsAdvect.hpp:601
//   ConstSparseIterator over getDomain() lsReduce.hpp:103, lsToMesh.hpp:87-116
//   Domain::insertPoints, finalize       lsDomain.hpp:117, :135
//   PointData accessors                  lsBooleanOperation.hpp:160-164
// A D = 2 domain becomes a LevelSet with grid.dim = 2 and the third index of
// every point and run start 0 (the layout vlsg_set_grid documents).
#pragma once

#include <hrleSparseIterator.hpp>
#include <lsDomain.hpp>

#include "vlsgAdvect.hpp"

namespace vlsg {

// The points (HRLE order), undefined runs, width and scalar point data of a
// viennals::Domain.
template <class T, int D> LevelSet toVlsg(const viennals::Domain<T, D> &d) {
  static_assert(D == 2 || D == 3, "D = 2 or 3");
  LevelSet ls;
  const auto &g = d.getGrid();
  ls.grid.dim = D;
  for (int i = 0; i < D; ++i) {
    ls.grid.min[i] = g.getMinIndex(i);
    ls.grid.max[i] = g.getMaxIndex(i);
    ls.grid.boundary[i] = (int32_t)g.getBoundaryConditions(i);
  }
  ls.grid.gridDelta = g.getGridDelta();
  for (viennahrle::ConstSparseIterator<typename viennals::Domain<T, D>::DomainType> it(
           d.getDomain());
       !it.isFinished(); ++it) {
    const auto idx = it.getStartIndices();
    const int32_t x = (int32_t)idx[0], y = (int32_t)idx[1], z = D == 3 ? (int32_t)idx[D - 1] : 0;
    if (it.isDefined()) {
      ls.indices.insert(ls.indices.end(), {x, y, z});
      ls.values.push_back((double)it.getValue());
    } else {
      ls.runStart.insert(ls.runStart.end(), {x, y, z});
      ls.runSign.push_back(it.getValue() < 0 ? -1 : 1);
    }
  }
  ls.width = d.getLevelSetWidth();
  const auto &pd = d.getPointData(); // scalar arrays, one value per defined point
  for (unsigned i = 0; i < pd.getScalarDataSize(); ++i) {
    const auto *a = pd.getScalarData(i);
    ls.pointData[pd.getScalarDataLabel(i)] = std::vector<double>(a->begin(), a->end());
  }
  return ls;
}

// Refill a viennals::Domain from a LevelSet (points in HRLE order, as apply()
// writes them back); HRLE rebuilds the undefined runs from the points' signs.
template <class T, int D> void fromVlsg(const LevelSet &ls, viennals::Domain<T, D> &d) {
  static_assert(D == 2 || D == 3, "D = 2 or 3");
  typename viennals::Domain<T, D>::PointValueVectorType pts;
  pts.reserve(ls.values.size());
  for (size_t i = 0; i < ls.values.size(); ++i) {
    viennahrle::Index<D> idx;
    for (int k = 0; k < D; ++k) idx[k] = ls.indices[3 * i + k];
    pts.emplace_back(idx, T(ls.values[i]));
  }
  d.insertPoints(pts, false); // the points arrive in HRLE order
  d.getDomain().segment();
  d.finalize(ls.width);
  d.getPointData().clear();
  for (const auto &kv : ls.pointData)
    d.getPointData().insertNextScalarData(std::vector<T>(kv.second.begin(), kv.second.end()),
                                          kv.first);
}

} // namespace vlsg
