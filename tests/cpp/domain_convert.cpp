// Drives include/vlsgViennaLS.hpp against the ViennaLS/HRLE stand-ins in
// tests/cpp/viennals_stub: reads a level set (grid, points and undefined runs
// in HRLE order), builds a viennals::Domain<double,D> of it with a point-data
// array "ids" (0, 1, ...), converts it with toVlsg, and either
//   roundtrip : converts it straight back with fromVlsg, or
//   advect N  : runs N single steps of vlsg::Advect<double> (LAX_FRIEDRICHS_1ST_ORDER
//               for D = 2, ENGQUIST_OSHER_1ST_ORDER for D = 3; scalar velocity
//               `rate`, FE) on the GPU and converts the result back,
// then writes what the Domain holds.  Input: int32 dim; int64 min[dim],
// max[dim]; int32 boundary[dim]; double gridDelta, rate; int64 n;
// int32 idx[3n] (third 0 for D = 2); double values[n]; int64 m;
// int32 runStart[3m]; int8 runSign[m]; int32 width.  Output: int64 n;
// int32 idx[3n]; double values[n]; int32 width; double ids[n] (the "ids"
// point data after the conversions, in the same order); int32 segmented.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "vlsgViennaLS.hpp"

template <class V> static void readN(FILE *f, V *p, size_t n) {
  if (n && std::fread(p, sizeof(V), n, f) != n) std::exit(2);
}
template <class V> static void writeN(FILE *f, const V *p, size_t n) {
  if (n) std::fwrite(p, sizeof(V), n, f);
}

struct Input {
  int32_t dim = 3;
  int64_t lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  int32_t bc[3] = {1, 1, 1};
  double delta = 1, rate = 1;
  std::vector<int32_t> idx, rs;
  std::vector<double> val;
  std::vector<int8_t> sg;
  int32_t width = 2;
};

static long long key(const int32_t *p) {
  return ((long long)(p[2] + (1 << 21)) << 44) + ((long long)(p[1] + (1 << 21)) << 22) +
         (long long)(p[0] + (1 << 21));
}

template <int D> static int run(const Input &in, const char *mode, int steps, FILE *out) {
  viennals::Domain<double, D> dom;
  for (int i = 0; i < D; ++i) {
    dom.grid.lo[i] = in.lo[i];
    dom.grid.hi[i] = in.hi[i];
    dom.grid.bc[i] = (viennahrle::BoundaryType)in.bc[i];
  }
  dom.grid.delta = in.delta;
  // points and run starts merged in HRLE order
  const size_t n = in.val.size(), m = in.sg.size();
  size_t a = 0, b = 0;
  while (a < n || b < m) {
    const bool point = b >= m || (a < n && key(&in.idx[3 * a]) < key(&in.rs[3 * b]));
    typename viennals::Domain<double, D>::DomainType::Entry e;
    const int32_t *p = point ? &in.idx[3 * a] : &in.rs[3 * b];
    for (int k = 0; k < D; ++k) e.start[k] = p[k];
    e.defined = point;
    e.value = point ? in.val[a] : (in.sg[b] < 0 ? -std::numeric_limits<double>::max()
                                                 : std::numeric_limits<double>::max());
    dom.domain.entries.push_back(e);
    (point ? a : b)++;
  }
  dom.finalize(in.width);
  std::vector<double> ids(n);
  for (size_t i = 0; i < n; ++i) ids[i] = (double)i;
  dom.getPointData().insertNextScalarData(ids, "ids");

  vlsg::LevelSet ls = vlsg::toVlsg(dom);
  if (ls.grid.dim != D || ls.values.size() != n || ls.runSign.size() != m) return 3;
  if (std::strcmp(mode, "advect") == 0) {
    auto shared = std::make_shared<vlsg::LevelSet>(std::move(ls));
    auto vel = std::make_shared<vlsg::VelocityFunctor>(1);
    vel->rate(0, in.rate);
    vlsg::Advect<double> adv;
    adv.insertNextLevelSet(shared);
    adv.setVelocityField(vel);
    adv.setSpatialScheme(D == 2 ? vlsg::SpatialSchemeEnum::LAX_FRIEDRICHS_1ST_ORDER
                                : vlsg::SpatialSchemeEnum::ENGQUIST_OSHER_1ST_ORDER);
    adv.setUpdatePointData(true);
    for (int s = 0; s < steps; ++s) adv.apply();
    ls = *shared;
  }
  viennals::Domain<double, D> back;
  vlsg::fromVlsg(ls, back);
  const int64_t nOut = (int64_t)back.getDomain().getNumberOfPoints();
  writeN(out, &nOut, 1);
  std::vector<int32_t> idx;
  std::vector<double> val;
  for (viennahrle::ConstSparseIterator<typename viennals::Domain<double, D>::DomainType> it(
           back.getDomain());
       !it.isFinished(); ++it) {
    if (!it.isDefined()) continue;
    for (int k = 0; k < 3; ++k) idx.push_back(k < D ? (int32_t)it.getStartIndices(k) : 0);
    val.push_back(it.getValue());
  }
  writeN(out, idx.data(), idx.size());
  writeN(out, val.data(), val.size());
  const int32_t w = back.getLevelSetWidth();
  writeN(out, &w, 1);
  const auto &pd = back.getPointData();
  std::vector<double> outIds(nOut, -2.0);
  for (unsigned i = 0; i < pd.getScalarDataSize(); ++i)
    if (pd.getScalarDataLabel(i) == "ids" && (int64_t)pd.getScalarData(i)->size() == nOut)
      outIds = *pd.getScalarData(i);
  writeN(out, outIds.data(), outIds.size());
  const int32_t seg = back.getDomain().segmented;
  writeN(out, &seg, 1);
  return 0;
}

int main(int argc, char **argv) {
  if (argc < 4) return 1;
  FILE *f = std::fopen(argv[1], "rb");
  if (!f) return 1;
  Input in;
  readN(f, &in.dim, 1);
  readN(f, in.lo, in.dim);
  readN(f, in.hi, in.dim);
  readN(f, in.bc, in.dim);
  readN(f, &in.delta, 1);
  readN(f, &in.rate, 1);
  int64_t n = 0, m = 0;
  readN(f, &n, 1);
  in.idx.resize(3 * n);
  in.val.resize(n);
  readN(f, in.idx.data(), 3 * n);
  readN(f, in.val.data(), n);
  readN(f, &m, 1);
  in.rs.resize(3 * m);
  in.sg.resize(m);
  readN(f, in.rs.data(), 3 * m);
  readN(f, in.sg.data(), m);
  readN(f, &in.width, 1);
  std::fclose(f);
  FILE *out = std::fopen(argv[2], "wb");
  if (!out) return 1;
  const int steps = argc > 4 ? std::atoi(argv[4]) : 0;
  const int rc = in.dim == 2 ? run<2>(in, argv[3], steps, out) : run<3>(in, argv[3], steps, out);
  std::fclose(out);
  return rc;
}
