// Test stand-in for ViennaHRLE's sparse iterator and domain: the names and
// call signatures include/vlsgViennaLS.hpp uses, as the reference calls them
// (lsReduce.hpp:103, lsToMesh.hpp:87-116, lsFromSurfaceMesh.hpp:281-282,
// lsDomain.hpp:32-34), over a flat list of entries in HRLE order.  It checks
// that the conversions compile against those signatures and convert
// correctly; it is not ViennaHRLE.
#pragma once

#include <array>
#include <cstddef>
#include <vector>

namespace viennahrle {

template <int D> struct Index {
  std::array<long long, D> v{};
  long long &operator[](int i) { return v[i]; }
  long long operator[](int i) const { return v[i]; }
};

enum class BoundaryType : unsigned { REFLECTIVE_BOUNDARY = 0, INFINITE_BOUNDARY = 1,
                                     PERIODIC_BOUNDARY = 2, POS_INFINITE_BOUNDARY = 3,
                                     NEG_INFINITE_BOUNDARY = 4 };

template <int D> struct Grid {
  std::array<long long, D> lo{}, hi{};
  std::array<BoundaryType, D> bc{};
  double delta = 1.0;
  long long getMinIndex(int i) const { return lo[i]; }
  long long getMaxIndex(int i) const { return hi[i]; }
  BoundaryType getBoundaryConditions(int i) const { return bc[i]; }
  double getGridDelta() const { return delta; }
};

// Entries in HRLE order: defined points and the starts of undefined runs.
template <class T, int D> struct Domain {
  struct Entry {
    Index<D> start;
    T value;
    bool defined;
  };
  std::vector<Entry> entries;
  int segmented = 0;
  void segment() { ++segmented; }
  std::size_t getNumberOfPoints() const {
    std::size_t n = 0;
    for (const auto &e : entries) n += e.defined;
    return n;
  }
};

template <class DomainT> class ConstSparseIterator {
  const DomainT &d;
  std::size_t i = 0;

public:
  explicit ConstSparseIterator(const DomainT &domain) : d(domain) {}
  bool isFinished() const { return i >= d.entries.size(); }
  ConstSparseIterator &operator++() {
    ++i;
    return *this;
  }
  bool isDefined() const { return d.entries[i].defined; }
  auto getValue() const { return d.entries[i].value; }
  auto getStartIndices() const { return d.entries[i].start; }
  long long getStartIndices(int k) const { return d.entries[i].start[k]; }
};

} // namespace viennahrle
