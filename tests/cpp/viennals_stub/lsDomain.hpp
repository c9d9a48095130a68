// Test stand-in for viennals::Domain (lsDomain.hpp:27-269) and its point
// data: the members include/vlsgViennaLS.hpp calls, with the reference's
// names and types (DomainType, PointValueVectorType, getGrid, getDomain,
// insertPoints, finalize, getLevelSetWidth, getPointData; the point data's
// scalar accessors as lsBooleanOperation.hpp:160-164 calls them).
// insertPoints stores the points as defined entries without rebuilding
// undefined runs (ViennaHRLE's FillDomainWithSignedDistance does that).
#pragma once

#include <limits>
#include <string>
#include <utility>
#include <vector>

#include "hrleSparseIterator.hpp"

namespace viennals {

template <class T> struct PointData {
  std::vector<std::vector<T>> data;
  std::vector<std::string> labels;
  unsigned getScalarDataSize() const { return (unsigned)data.size(); }
  const std::vector<T> *getScalarData(unsigned i) const { return &data[i]; }
  std::string getScalarDataLabel(unsigned i) const { return labels[i]; }
  void insertNextScalarData(std::vector<T> v, std::string label) {
    data.push_back(std::move(v));
    labels.push_back(std::move(label));
  }
  void clear() { data.clear(), labels.clear(); }
};

template <class T, int D> class Domain {
public:
  typedef viennahrle::Domain<T, D> DomainType;
  typedef viennahrle::Grid<D> GridType;
  typedef std::vector<std::pair<viennahrle::Index<D>, T>> PointValueVectorType;

  GridType grid;
  DomainType domain;
  int levelSetWidth = 1;
  PointData<T> pointData;

  const GridType &getGrid() const { return grid; }
  DomainType &getDomain() { return domain; }
  const DomainType &getDomain() const { return domain; }
  int getLevelSetWidth() const { return levelSetWidth; }
  void finalize(int newWidth) { levelSetWidth = newWidth; }
  PointData<T> &getPointData() { return pointData; }
  const PointData<T> &getPointData() const { return pointData; }
  void insertPoints(PointValueVectorType pts, bool /*sort*/ = true) {
    domain.entries.clear();
    for (auto &p : pts) domain.entries.push_back({p.first, p.second, true});
  }
};

} // namespace viennals
