// vlsgAdvect.hpp -- header-only C++ front of libvlsgpu with the interface of
// viennals::Advect<T,D> (include/viennals/lsAdvect.hpp:836-1043 of ViennaLS
// 5.8.3): the same setters and getters, level sets inserted bottom to top,
// apply() writing the results back into the same level-set objects, and
// errors logged and swallowed like VIENNACORE_LOG_ERROR + return.
//
// `vlsg::LevelSet` holds what crosses the C ABI for one level set: the grid,
// the defined points with their values (grid units) and the undefined runs,
// all in HRLE order (what a viennahrle::ConstSparseIterator over a
// viennals::Domain<T,3> visits: defined points and undefined runs).
#pragma once

#include <array>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "vlsg.h"

namespace vlsg {

enum class SpatialSchemeEnum : unsigned {
  ENGQUIST_OSHER_1ST_ORDER = 0,
  ENGQUIST_OSHER_2ND_ORDER = 1,
  LAX_FRIEDRICHS_1ST_ORDER = 2,
  LAX_FRIEDRICHS_2ND_ORDER = 3,
  LOCAL_LAX_FRIEDRICHS_ANALYTICAL_1ST_ORDER = 4,
  LOCAL_LOCAL_LAX_FRIEDRICHS_1ST_ORDER = 5,
  LOCAL_LOCAL_LAX_FRIEDRICHS_2ND_ORDER = 6,
  LOCAL_LAX_FRIEDRICHS_1ST_ORDER = 7,
  LOCAL_LAX_FRIEDRICHS_2ND_ORDER = 8,
  STENCIL_LOCAL_LAX_FRIEDRICHS_1ST_ORDER = 9,
  WENO_3RD_ORDER = 10,
  WENO_5TH_ORDER = 11
};
enum class TemporalSchemeEnum : unsigned {
  FORWARD_EULER = 0,
  RUNGE_KUTTA_2ND_ORDER = 1,
  RUNGE_KUTTA_3RD_ORDER = 2
};

struct Grid {
  std::array<int64_t, 3> min{}, max{};
  std::array<int32_t, 3> boundary{VLSG_INFINITE_BOUNDARY, VLSG_INFINITE_BOUNDARY,
                                   VLSG_INFINITE_BOUNDARY};
  double gridDelta = 1.0;
  // 2 for Advect<T,2>: min, max and boundary use their first two entries, and
  // the indices of the level sets keep 3 per point with the third 0
  int dim = 3;
};

struct LevelSet {
  Grid grid;
  std::vector<int32_t> indices; // 3 per point, HRLE order
  std::vector<double> values;
  std::vector<int32_t> runStart; // 3 per undefined run
  std::vector<int8_t> runSign;
  int width = 2;
  // Version stamp: Advect::apply writes its results back with a fresh stamp
  // and keeps the device copy; a later apply on the same, unchanged objects
  // skips the upload.  Code that changes a level set in place afterwards
  // calls touch() (a new object, or one whose array sizes changed, is always
  // uploaded).
  uint64_t version = 0;
  void touch() { version = 0; }
  // Domain::getPointData(): scalar arrays per defined point, by label.  The
  // top level set's arrays are carried through Advect::apply the way the
  // reference's passes translate them (setSaveAdvectionVelocities adds
  // "AdvectionVelocities" and "Dissipation"; setUpdatePointData(false)
  // drops them all).
  std::map<std::string, std::vector<double>> pointData;
  int64_t numberOfPoints() const { return (int64_t)values.size(); }
};

// Stamps for LevelSet::version (one counter for every front).
inline uint64_t freshLevelSetStamp() {
  static std::atomic<uint64_t> next{1};
  return next.fetch_add(1);
}

// Device velocity field: per-material polynomial in the normal (vlsg.h).
struct VelocityFunctor {
  vlsg_velocity_desc desc{};
  explicit VelocityFunctor(int materials = 1) { desc.n_materials = materials; }
  VelocityFunctor &rate(int m, double v) { desc.rate[m] = v; return *this; }
  VelocityFunctor &linear(int m, int k, double pos, double neg) {
    desc.lin_pos[m][k] = pos, desc.lin_neg[m][k] = neg;
    return *this;
  }
  VelocityFunctor &absolute(int m, int k, double pos, double neg) {
    desc.abs_pos[m][k] = pos, desc.abs_neg[m][k] = neg;
    return *this;
  }
  VelocityFunctor &square(int m, int k, double pos, double neg) {
    desc.sq_pos[m][k] = pos, desc.sq_neg[m][k] = neg;
    return *this;
  }
  VelocityFunctor &dissipationAlpha(int m, int dir, double a) {
    desc.alpha[m][dir] = a;
    return *this;
  }
  VelocityFunctor &vector(int m, double x, double y, double z) {
    desc.vec[m][0] = x, desc.vec[m][1] = y, desc.vec[m][2] = z;
    return *this;
  }
};

// viennals::VelocityField<T> (lsVelocityField.hpp:11-41) for user code: the
// library asks it through its host callback, in batches of points and from
// several threads at once (as the reference calls it from OpenMP threads,
// lsAdvect.hpp:464), so overrides must be thread-safe.  The coordinate is
// index * gridDelta, the point id the point's rank among the defined points
// of the expanded top level set in HRLE order.
template <class T> class VelocityField {
public:
  virtual ~VelocityField() = default;
  virtual T getScalarVelocity(const std::array<T, 3> & /*coordinate*/, int /*material*/,
                              const std::array<T, 3> & /*normalVector*/,
                              unsigned long /*pointId*/) {
    return 0;
  }
  virtual std::array<T, 3> getVectorVelocity(const std::array<T, 3> & /*coordinate*/,
                                             int /*material*/,
                                             const std::array<T, 3> & /*normalVector*/,
                                             unsigned long /*pointId*/) {
    return {0, 0, 0};
  }

  // asked by LOCAL_LAX_FRIEDRICHS_ANALYTICAL_1ST_ORDER (lsVelocityField.hpp:35-38)
  virtual T getDissipationAlpha(int /*direction*/, int /*material*/,
                                const std::array<T, 3> & /*centralDifferences*/) {
    return 0;
  }

  // vlsg_alpha_cb trampoline (user = the field)
  static int alphaCallback(void *user, int64_t n, const int32_t *directions,
                           const int32_t *materials, const double *cd, double *alphaOut) {
    auto *f = static_cast<VelocityField<T> *>(user);
    try {
      for (int64_t i = 0; i < n; ++i) {
        const std::array<T, 3> c{T(cd[3 * i]), T(cd[3 * i + 1]), T(cd[3 * i + 2])};
        alphaOut[i] = (double)f->getDissipationAlpha(directions[i], materials[i], c);
      }
    } catch (...) {
      return 1;
    }
    return 0;
  }

  // vlsg_velocity_cb trampoline (user = the field)
  static int callback(void *user, int64_t n, const double *coords, const int32_t *materials,
                      const double *normals, const uint64_t *pointIds, double *scalarOut,
                      double *vectorOut) {
    auto *f = static_cast<VelocityField<T> *>(user);
    try {
      for (int64_t i = 0; i < n; ++i) {
        const std::array<T, 3> c{T(coords[3 * i]), T(coords[3 * i + 1]), T(coords[3 * i + 2])};
        const std::array<T, 3> nv{T(normals[3 * i]), T(normals[3 * i + 1]), T(normals[3 * i + 2])};
        const unsigned long id = (unsigned long)pointIds[i];
        scalarOut[i] = (double)f->getScalarVelocity(c, materials[i], nv, id);
        const std::array<T, 3> v = f->getVectorVelocity(c, materials[i], nv, id);
        for (int k = 0; k < 3; ++k) vectorOut[3 * i + k] = (double)v[k];
      }
    } catch (...) {
      return 1;
    }
    return 0;
  }
};

template <class T> class Advect {
  std::vector<std::shared_ptr<LevelSet>> levelSets;
  std::shared_ptr<VelocityFunctor> velocities;
  std::shared_ptr<VelocityField<T>> field; // host callback mode when set
  std::function<bool(std::shared_ptr<LevelSet>)> velocityUpdateCallback;
  static int updateTrampoline(void *user, const vlsg_levelset_view *v) {
    auto *self = static_cast<Advect<T> *>(user);
    auto ls = std::make_shared<LevelSet>();
    ls->grid = self->levelSets.back()->grid;
    ls->indices.assign(v->indices, v->indices + 3 * v->n_points);
    ls->values.assign(v->values, v->values + v->n_points);
    ls->runStart.assign(v->run_start, v->run_start + 3 * v->n_runs);
    ls->runSign.assign(v->run_sign, v->run_sign + v->n_runs);
    ls->width = v->width;
    try {
      self->velocityUpdateCallback(ls); // the reference ignores the bool
    } catch (...) {
      return 1;
    }
    return 0;
  }
  vlsg_advect_params params{};
  vlsg_advect_result result{};
  vlsg_context *ctx = nullptr;
  uint64_t skippedUploads = 0;
  int device = 0;

  static void logError(const std::string &m) { std::fprintf(stderr, "[vlsg] %s\n", m.c_str()); }
  bool check(int rc) {
    if (rc == VLSG_OK) return true;
    logError(vlsg_last_error(ctx));
    return false;
  }

public:
  // labels of the saved arrays (lsAdvect.hpp:833-834)
  static constexpr const char *velocityLabel = "AdvectionVelocities";
  static constexpr const char *dissipationLabel = "Dissipation";

  Advect() { vlsg_default_params(&params), result.current_time_step = -1.; }
  explicit Advect(std::shared_ptr<LevelSet> ls) : Advect() { levelSets.push_back(ls); }
  Advect(std::shared_ptr<LevelSet> ls, std::shared_ptr<VelocityFunctor> v) : Advect() {
    levelSets.push_back(ls);
    velocities = v;
  }
  Advect(std::vector<std::shared_ptr<LevelSet>> lss, std::shared_ptr<VelocityFunctor> v)
      : Advect() {
    levelSets = lss;
    velocities = v;
  }
  ~Advect() {
    if (ctx) vlsg_destroy(ctx);
  }
  Advect(const Advect &) = delete;
  Advect &operator=(const Advect &) = delete;

  void setDevice(int d) { device = d; }
  void insertNextLevelSet(std::shared_ptr<LevelSet> ls) { levelSets.push_back(ls); }
  void clearLevelSets() { levelSets.clear(); }
  void setVelocityField(std::shared_ptr<VelocityFunctor> v) { velocities = v, field.reset(); }
  void setVelocityField(std::shared_ptr<VelocityField<T>> f) { field = f, velocities.reset(); }
  void setAdvectionTime(double t) { params.advection_time = t; }
  void setSingleStep(bool b) { params.single_step = b; }
  void setTimeStepRatio(const double &cfl) { params.time_step_ratio = cfl; }
  void setCalculateNormalVectors(bool b) { params.calculate_normal_vectors = b; }
  void setIgnoreVoids(bool b) { params.ignore_voids = b; }
  void setAdaptiveTimeStepping(bool b = true, unsigned subdivisions = 20) {
    params.adaptive_time_stepping = b;
    params.adaptive_subdivisions = subdivisions < 1 ? 1 : subdivisions;
  }
  void setSaveAdvectionVelocities(bool b) { params.save_advection_velocities = b; }
  void setSpatialScheme(SpatialSchemeEnum s) { params.spatial_scheme = (int32_t)s; }
  // the deprecated name of setSpatialScheme (lsAdvect.hpp:940-946)
  void setIntegrationScheme(SpatialSchemeEnum s) { setSpatialScheme(s); }
  void setTemporalScheme(TemporalSchemeEnum s) { params.temporal_scheme = (int32_t)s; }
  void setDissipationAlpha(const double &a) { params.dissipation_alpha = a; }
  void setCheckDissipation(bool b) { params.check_dissipation = b; }
  void setUpdatePointData(bool b) { params.update_point_data = b; }
  // StencilLocalLaxFriedrichsScalar<T,D,1>::setMaxDissipation, per Advect here
  void setMaxDissipation(double d) { params.max_dissipation = d; }
  // lsAdvect.hpp:966-969: called between RK2/RK3 stages with a copy of the
  // top level set
  void setVelocityUpdateCallback(std::function<bool(std::shared_ptr<LevelSet>)> cb) {
    velocityUpdateCallback = std::move(cb);
  }

  double getAdvectedTime() const { return result.advected_time; }
  double getCurrentTimeStep() const { return result.current_time_step; }
  unsigned getNumberOfTimeSteps() const { return result.number_of_time_steps; }
  double getTimeStepRatio() const { return params.time_step_ratio; }
  bool getCalculateNormalVectors() const { return params.calculate_normal_vectors; }
  const vlsg_advect_result &getResult() const { return result; }

  // Advect::apply, lsAdvect.hpp:1017-1043
  // Advect::prepareLS (lsAdvect.hpp:972-1015): the top level set expanded to
  // the width the spatial scheme reads, written back.
  void prepareLS() {
    if (levelSets.empty()) return logError("No level sets passed to Advect.");
    if (!uploadLevelSets()) return;
    if (!check(vlsg_prepare_ls(ctx, params.spatial_scheme))) return;
    if (downloadLevelSet(levelSets.size() - 1)) markResident();
  }

  void apply() {
    if (levelSets.empty()) return logError("No level sets passed to Advect. Not advecting.");
    if (!velocities && !field)
      return logError("No velocity field passed to Advect. Not advecting.");
    const bool save = params.save_advection_velocities != 0;
    const bool track = save || !levelSets.back()->pointData.empty();
    params.track_point_data = track;
    if (!uploadLevelSets()) return;
    if (field) {
      if (!check(vlsg_set_velocity_callback(ctx, &VelocityField<T>::callback, field.get()))) return;
      if (!check(vlsg_set_dissipation_alpha_callback(ctx, &VelocityField<T>::alphaCallback,
                                                     field.get())))
        return;
    } else if (!check(vlsg_set_velocity_functor(ctx, &velocities->desc))) {
      return;
    }
    if (!check(vlsg_set_velocity_update_callback(
            ctx, velocityUpdateCallback ? &Advect<T>::updateTrampoline : nullptr, this)))
      return;
    if (!check(vlsg_advect(ctx, &params, &result))) return;
    for (size_t i = 0; i < levelSets.size(); ++i)
      if (!downloadLevelSet(i)) return;
    if (track && !translatePointData(save)) return;
    markResident();
  }

  // applies (and prepareLS calls) that found the device copy current
  uint64_t getSkippedUploads() const { return skippedUploads; }

private:
  // What the device holds since the last write-back: the level-set objects,
  // their stamps and array sizes (B2 of the drop-in contract: device state is
  // reused only while the host objects are unchanged).
  struct Resident {
    const LevelSet *ls;
    uint64_t version;
    size_t points, runs;
  };
  std::vector<Resident> resident;
  static uint64_t freshStamp() { return freshLevelSetStamp(); }
  bool residentUnchanged() const {
    if (!ctx || resident.size() != levelSets.size()) return false;
    for (size_t i = 0; i < levelSets.size(); ++i) {
      const LevelSet &ls = *levelSets[i];
      const Resident &r = resident[i];
      if (r.ls != &ls || ls.version == 0 || r.version != ls.version ||
          r.points != ls.values.size() || r.runs != ls.runSign.size())
        return false;
    }
    return true;
  }
  void markResident() {
    resident.clear();
    for (auto &p : levelSets) {
      p->version = freshStamp();
      resident.push_back({p.get(), p->version, p->values.size(), p->runSign.size()});
    }
  }

  // the context (created on first use) holding the grid and all level sets;
  // nothing crosses PCIe when the device copy is still current
  bool uploadLevelSets() {
    if (residentUnchanged()) {
      ++skippedUploads;
      return true;
    }
    resident.clear();
    if (!ctx) {
      const int precision = sizeof(T) == 4 ? VLSG_FP32 : VLSG_FP64;
      if (!check(vlsg_create(&ctx, device, precision))) return false;
    }
    const Grid &g = levelSets.back()->grid;
    if (!check(vlsg_set_grid(ctx, g.dim, g.min.data(), g.max.data(), g.boundary.data(), g.gridDelta)))
      return false;
    if (!check(vlsg_set_level_set_count(ctx, (int32_t)levelSets.size()))) return false;
    for (size_t i = 0; i < levelSets.size(); ++i) {
      const LevelSet &ls = *levelSets[i];
      if (!check(vlsg_upload_levelset(ctx, (int32_t)i, ls.numberOfPoints(), ls.indices.data(),
                                      ls.values.data(), (int64_t)ls.runSign.size(),
                                      ls.runStart.data(), ls.runSign.data(), ls.width)))
        return false;
    }
    return true;
  }
  // The top level set's point data after an advection: every array gathered
  // by the source ids (0 where there is none); the saved velocity arrays
  // replace earlier ones.
  bool translatePointData(bool save) {
    LevelSet &ls = *levelSets.back();
    const int64_t n = ls.numberOfPoints();
    std::vector<int64_t> src(n);
    std::vector<double> vel(n), diss(n);
    int32_t has = 0;
    if (!check(vlsg_download_point_data(ctx, (int32_t)levelSets.size() - 1, n, src.data(),
                                        vel.data(), diss.data(), &has)))
      return false;
    std::map<std::string, std::vector<double>> out;
    if (has) {
      for (auto &kv : ls.pointData) {
        if (save && (kv.first == velocityLabel || kv.first == dissipationLabel)) continue;
        std::vector<double> a(n, 0.0);
        for (int64_t i = 0; i < n; ++i)
          if (src[i] >= 0 && src[i] < (int64_t)kv.second.size()) a[i] = kv.second[src[i]];
        out[kv.first] = std::move(a);
      }
      if (save) {
        out[velocityLabel] = std::move(vel);
        out[dissipationLabel] = std::move(diss);
      }
    }
    ls.pointData = std::move(out);
    return true;
  }

  // level set i written back: defined points and undefined runs in HRLE
  // order, both built on the device
  bool downloadLevelSet(size_t i) {
    LevelSet &ls = *levelSets[i];
    int64_t n = 0;
    if (!check(vlsg_count_points(ctx, (int32_t)i, &n))) return false;
    ls.indices.resize(3 * n);
    ls.values.resize(n);
    int32_t w = 0;
    if (!check(vlsg_download_levelset(ctx, (int32_t)i, n, ls.indices.data(), ls.values.data(), &w)))
      return false;
    ls.width = w;
    int64_t m = 0;
    const int rc = vlsg_download_runs(ctx, (int32_t)i, 0, nullptr, nullptr, &m);
    if (rc != VLSG_OK && rc != VLSG_ERR_CAPACITY && !check(rc)) return false;
    ls.runStart.resize(3 * m);
    ls.runSign.resize(m);
    return check(vlsg_download_runs(ctx, (int32_t)i, m, ls.runStart.data(), ls.runSign.data(), &m));
  }
};

// The batching form for C++ callers: many independent domains, one level set
// and one device velocity functor each, advanced together in one context
// (vlsg_batch_*: every pass of a time step one kernel launch over all of
// them).  It replaces a loop over one Advect per domain (the style of
// examples/SquareEtch/SquareEtch.cpp:189-229); each apply() is one time step
// of every domain and writes the results back into the same LevelSet
// objects, with the getters per domain.  The domains stay on the device
// between applies while the objects are unchanged (version stamps, as
// Advect; a changed velocity functor sets the domains up again).  Limits as
// vlsg_batch_set_domains: periodic in x and y with
// extents in whole bricks of 8 points, infinite in z.
template <class T> class AdvectBatch {
  std::vector<std::shared_ptr<LevelSet>> domains;
  std::vector<std::shared_ptr<VelocityFunctor>> velocities;
  vlsg_advect_params params{};
  std::vector<vlsg_advect_result> results;
  vlsg_context *ctx = nullptr;
  int device = 0;
  struct Resident {
    const LevelSet *ls;
    uint64_t version;
    vlsg_velocity_desc vel; // the velocity the device copy was set up with
  };
  std::vector<Resident> resident;
  uint64_t skippedUploads = 0;

  static void logError(const std::string &m) { std::fprintf(stderr, "[vlsg] %s\n", m.c_str()); }
  bool check(int rc) {
    if (rc == VLSG_OK) return true;
    logError(vlsg_last_error(ctx));
    return false;
  }
  bool residentUnchanged() const {
    if (!ctx || resident.size() != domains.size()) return false;
    for (size_t d = 0; d < domains.size(); ++d)
      if (resident[d].ls != domains[d].get() || domains[d]->version == 0 ||
          resident[d].version != domains[d]->version ||
          std::memcmp(&resident[d].vel, &velocities[d]->desc, sizeof(vlsg_velocity_desc)) != 0)
        return false;
    return true;
  }
  bool upload() {
    if (!ctx && !check(vlsg_create(&ctx, device, sizeof(T) == 4 ? VLSG_FP32 : VLSG_FP64)))
      return false;
    if (residentUnchanged()) {
      ++skippedUploads;
      return true;
    }
    std::vector<vlsg_batch_domain> b(domains.size());
    for (size_t d = 0; d < domains.size(); ++d) {
      const LevelSet &ls = *domains[d];
      b[d] = vlsg_batch_domain{ls.grid.min.data(),   ls.grid.max.data(),  ls.grid.boundary.data(),
                               ls.grid.gridDelta,    ls.numberOfPoints(), ls.indices.data(),
                               ls.values.data(),     (int64_t)ls.runSign.size(),
                               ls.runStart.data(),   ls.runSign.data(),   ls.width,
                               &velocities[d]->desc};
    }
    return check(vlsg_batch_set_domains(ctx, (int32_t)b.size(), b.data()));
  }
  bool download(size_t d) {
    LevelSet &ls = *domains[d];
    int64_t n = 0;
    if (!check(vlsg_batch_count_points(ctx, (int32_t)d, &n))) return false;
    ls.indices.resize(3 * n);
    ls.values.resize(n);
    int32_t w = 0;
    if (!check(vlsg_batch_download(ctx, (int32_t)d, n, ls.indices.data(), ls.values.data(), &w)))
      return false;
    ls.width = w;
    int64_t m = 0;
    const int rc = vlsg_batch_download_runs(ctx, (int32_t)d, 0, nullptr, nullptr, &m);
    if (rc != VLSG_OK && rc != VLSG_ERR_CAPACITY && !check(rc)) return false;
    ls.runStart.resize(3 * m);
    ls.runSign.resize(m);
    return check(vlsg_batch_download_runs(ctx, (int32_t)d, m, ls.runStart.data(), ls.runSign.data(), &m));
  }

public:
  AdvectBatch() { vlsg_default_params(&params); }
  AdvectBatch(const AdvectBatch &) = delete;
  AdvectBatch &operator=(const AdvectBatch &) = delete;
  ~AdvectBatch() {
    if (ctx) vlsg_destroy(ctx);
  }
  void setDevice(int d) { device = d; }
  void insertNextDomain(std::shared_ptr<LevelSet> ls, std::shared_ptr<VelocityFunctor> v) {
    domains.push_back(std::move(ls));
    velocities.push_back(std::move(v));
  }
  void clearDomains() { domains.clear(), velocities.clear(), resident.clear(); }
  void setTimeStepRatio(const double &cfl) { params.time_step_ratio = cfl; }
  void setCalculateNormalVectors(bool b) { params.calculate_normal_vectors = b; }
  void setAdaptiveTimeStepping(bool b = true, unsigned subdivisions = 20) {
    params.adaptive_time_stepping = b;
    params.adaptive_subdivisions = subdivisions < 1 ? 1 : subdivisions;
  }
  void setSpatialScheme(SpatialSchemeEnum s) { params.spatial_scheme = (int32_t)s; }
  void setTemporalScheme(TemporalSchemeEnum s) { params.temporal_scheme = (int32_t)s; }
  void setDissipationAlpha(const double &a) { params.dissipation_alpha = a; }
  void setCheckDissipation(bool b) { params.check_dissipation = b; }

  // one time step of every domain, results written back
  void apply() {
    if (domains.empty()) return logError("No domains passed to AdvectBatch.");
    for (auto &v : velocities)
      if (!v) return logError("No velocity field passed to AdvectBatch.");
    for (auto &d : domains)
      if (d->grid.dim != 3) return logError("AdvectBatch: three-dimensional domains only.");
    if (!upload()) return;
    results.assign(domains.size(), vlsg_advect_result{});
    params.advection_time = 0.;
    if (!check(vlsg_batch_advect(ctx, &params, results.data()))) return;
    resident.clear();
    for (size_t d = 0; d < domains.size(); ++d) {
      if (!download(d)) return;
      domains[d]->version = freshLevelSetStamp();
      resident.push_back(Resident{domains[d].get(), domains[d]->version, velocities[d]->desc});
    }
  }
  double getAdvectedTime(size_t d) const { return results.at(d).advected_time; }
  double getCurrentTimeStep(size_t d) const { return results.at(d).current_time_step; }
  uint64_t getPointUpdates(size_t d) const { return results.at(d).point_updates; }
  // applies that found every domain's device copy current
  uint64_t getSkippedUploads() const { return skippedUploads; }
};

} // namespace vlsg
