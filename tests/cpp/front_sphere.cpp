// Drives libvlsgpu through the C++ front (include/vlsgAdvect.hpp) the way a
// ViennaLS user drives viennals::Advect: a sphere (MakeGeometry::makeSphere's
// distance rule, lsMakeGeometry.hpp:177-241) grown with a constant scalar
// velocity -- the device functor, or with a second argument "callback" the
// same velocity as a host VelocityField.  Prints steps, advected time, point
// count and a checksum.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <limits>
#include <string>

#include "vlsgAdvect.hpp"

struct UnitVelocity : vlsg::VelocityField<double> {
  double getScalarVelocity(const std::array<double, 3> &, int, const std::array<double, 3> &,
                           unsigned long) override {
    return 1.0;
  }
};

int main(int argc, char **argv) {
  const double gd = 0.25, radius = 5.0;
  auto ls = std::make_shared<vlsg::LevelSet>();
  ls->grid.gridDelta = gd;
  // makeSphere at the origin
  const int lo = (int)((0.0 - radius) / gd - 1), hi = (int)((0.0 + radius) / gd + 1);
  const double r2 = radius * radius, limit = 2.0 * 0.5 * gd + 1e-5;
  std::vector<std::array<int, 3>> undefStarts;
  for (int z = lo; z <= hi; ++z)
    for (int y = lo; y <= hi; ++y)
      for (int x = lo; x <= hi; ++x) {
        if (x == hi && y == hi && z == hi) continue;
        const int idx[3] = {x, y, z};
        double distance = std::numeric_limits<double>::max();
        for (int i = 0; i < 3; ++i) {
          const double yy = idx[(i + 1) % 3] * gd, zz = idx[(i + 2) % 3] * gd;
          const double xx = r2 - yy * yy - zz * zz;
          if (xx < 0.) continue;
          const double dr = std::abs(idx[i] * gd) - std::sqrt(xx);
          if (std::abs(dr) < std::abs(distance)) distance = dr;
        }
        if (std::abs(distance) <= limit) {
          ls->indices.insert(ls->indices.end(), {x, y, z});
          ls->values.push_back(distance / gd);
        }
      }
  // undefined runs: every undefined stretch of a row takes the sign of its
  // geometric inside/outside test
  const int32_t NI = -((1 << 20) - 2);
  ls->runStart.insert(ls->runStart.end(), {NI, NI, NI});
  ls->runSign.push_back(1);
  size_t p = 0;
  for (int z = lo; z <= hi; ++z)
    for (int y = lo; y <= hi; ++y) {
      bool prevDefined = false;
      for (int x = lo - 1; x <= hi + 1; ++x) {
        const bool defined = p < ls->values.size() && ls->indices[3 * p] == x &&
                             ls->indices[3 * p + 1] == y && ls->indices[3 * p + 2] == z;
        if (defined) {
          ++p;
        } else if (prevDefined || x == lo - 1) {
          const double s = (x * gd) * (x * gd) + (y * gd) * (y * gd) + (z * gd) * (z * gd);
          ls->runStart.insert(ls->runStart.end(), {x == lo - 1 ? NI : x, y, z});
          ls->runSign.push_back(s < r2 ? -1 : 1);
        }
        prevDefined = defined;
      }
    }
  ls->width = 2;

  auto vel = std::make_shared<vlsg::VelocityFunctor>(1);
  vel->rate(0, 1.0);
  vlsg::Advect<double> advect(ls, vel);
  if (argc > 2 && std::string(argv[2]) == "callback")
    advect.setVelocityField(std::make_shared<UnitVelocity>());
  advect.setSpatialScheme(vlsg::SpatialSchemeEnum::ENGQUIST_OSHER_1ST_ORDER);
  advect.setTemporalScheme(vlsg::TemporalSchemeEnum::FORWARD_EULER);
  advect.setTimeStepRatio(0.5);
  if (argc > 2 && std::string(argv[2]) == "loop") {
    // a caller that loops single steps (as the reference's examples loop
    // Advect::apply): argv[1] steps of advectionTime 0; the level set stays
    // on the device between them.  After the loop the object is changed in
    // place and touch()ed, so the next apply uploads it again.
    advect.setAdvectionTime(0.0);
    const int steps = argc > 1 ? std::atoi(argv[1]) : 5;
    for (int k = 0; k < steps; ++k) advect.apply();
    std::printf("skipped %llu ", (unsigned long long)advect.getSkippedUploads());
    for (auto &v : ls->values) v = std::min(v, 0.25) ; // change in place ...
    ls->touch();                                        // ... and say so
    advect.apply();
    std::printf("after_touch %llu ", (unsigned long long)advect.getSkippedUploads());
  } else {
    advect.setAdvectionTime(argc > 1 ? std::atof(argv[1]) : 2.0);
    advect.apply();
  }
  double sum = 0;
  for (size_t i = 0; i < ls->values.size(); ++i)
    sum += ls->values[i] * (1.0 + 1e-3 * (ls->indices[3 * i] + 7 * ls->indices[3 * i + 1] +
                                          13 * ls->indices[3 * i + 2]));
  std::printf("steps %u time %.17g points %lld width %d runs %zu checksum %.17g\n",
              advect.getNumberOfTimeSteps(), advect.getAdvectedTime(),
              (long long)ls->numberOfPoints(), ls->width, ls->runSign.size(), sum);
  return advect.getNumberOfTimeSteps() > 0 ? 0 : 1;
}
