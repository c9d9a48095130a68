// Drives the batching form through the C++ front (vlsg::AdvectBatch in
// include/vlsgAdvect.hpp): reads domains from a binary file, advances all of
// them `steps` time steps (LOCAL_LAX_FRIEDRICHS_1ST_ORDER, RK2, FP32) and
// writes every domain's level set and advected time back.  File layout, per
// domain: int64 min[3], max[3]; int32 boundary[3]; double gridDelta, rate;
// int64 n; int32 indices[3n]; double values[n]; int64 m; int32 runStart[3m];
// int8 runSign[m]; int32 width -- after an int32 domain count.  The output
// repeats the level-set part per domain, followed by double advectedTime.
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <vector>

#include "vlsgAdvect.hpp"

template <class V> static void readN(FILE *f, V *p, size_t n) {
  if (n && std::fread(p, sizeof(V), n, f) != n) std::exit(2);
}
template <class V> static void writeN(FILE *f, const V *p, size_t n) {
  if (n) std::fwrite(p, sizeof(V), n, f);
}

int main(int argc, char **argv) {
  if (argc < 4) return 1;
  FILE *in = std::fopen(argv[1], "rb");
  if (!in) return 1;
  const int steps = std::atoi(argv[3]);
  int32_t count = 0;
  readN(in, &count, 1);
  vlsg::AdvectBatch<float> batch;
  std::vector<std::shared_ptr<vlsg::LevelSet>> doms;
  for (int d = 0; d < count; ++d) {
    auto ls = std::make_shared<vlsg::LevelSet>();
    readN(in, ls->grid.min.data(), 3);
    readN(in, ls->grid.max.data(), 3);
    readN(in, ls->grid.boundary.data(), 3);
    double rate = 0;
    readN(in, &ls->grid.gridDelta, 1);
    readN(in, &rate, 1);
    int64_t n = 0, m = 0;
    readN(in, &n, 1);
    ls->indices.resize(3 * n);
    ls->values.resize(n);
    readN(in, ls->indices.data(), 3 * n);
    readN(in, ls->values.data(), n);
    readN(in, &m, 1);
    ls->runStart.resize(3 * m);
    ls->runSign.resize(m);
    readN(in, ls->runStart.data(), 3 * m);
    readN(in, ls->runSign.data(), m);
    readN(in, &ls->width, 1);
    auto v = std::make_shared<vlsg::VelocityFunctor>(1);
    v->rate(0, rate);
    batch.insertNextDomain(ls, v);
    doms.push_back(ls);
  }
  std::fclose(in);
  batch.setSpatialScheme(vlsg::SpatialSchemeEnum::LOCAL_LAX_FRIEDRICHS_1ST_ORDER);
  batch.setTemporalScheme(vlsg::TemporalSchemeEnum::RUNGE_KUTTA_2ND_ORDER);
  std::vector<double> time(count, 0.0);
  for (int s = 0; s < steps; ++s) {
    batch.apply();
    for (int d = 0; d < count; ++d) time[d] += batch.getAdvectedTime(d);
  }
  FILE *out = std::fopen(argv[2], "wb");
  if (!out) return 1;
  writeN(out, &count, 1);
  for (int d = 0; d < count; ++d) {
    const vlsg::LevelSet &ls = *doms[d];
    const int64_t n = ls.numberOfPoints(), m = (int64_t)ls.runSign.size();
    writeN(out, &n, 1);
    writeN(out, ls.indices.data(), 3 * n);
    writeN(out, ls.values.data(), n);
    writeN(out, &m, 1);
    writeN(out, ls.runStart.data(), 3 * m);
    writeN(out, ls.runSign.data(), m);
    writeN(out, &ls.width, 1);
    writeN(out, &time[d], 1);
  }
  std::fclose(out);
  std::printf("skipped %llu\n", (unsigned long long)batch.getSkippedUploads());
  return 0;
}
