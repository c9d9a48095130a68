// vlso_api.cpp -- TEST INFRASTRUCTURE ONLY: extern "C" surface of the oracle
// (FP64 CPU restatement of ViennaLS 5.8.3's advection path) for the ctypes
// wrapper in oracle/oracle.py.  Used by tests/, __graft_entry__.smoke() and
// the CPU-baseline leg of bench.py, never by the product library.
#include <memory>
#include <mutex>

#include <type_traits>

#include "vlso_advect.hpp"
#include "vlso_metrics.hpp"

namespace {
thread_local std::string g_err;

struct Handle {
  int D;
  std::unique_ptr<vlso::LS<2>> l2;
  std::unique_ptr<vlso::LS<3>> l3;
};

template <class F> int guarded(F f) {
  try {
    return f();
  } catch (const std::exception &e) {
    g_err = e.what();
    return -1;
  }
}

template <int D> vlso::LS<D> &get(Handle *h);
template <> vlso::LS<2> &get<2>(Handle *h) { return *h->l2; }
template <> vlso::LS<3> &get<3>(Handle *h) { return *h->l3; }

template <int D>
int64_t listPoints(vlso::LS<D> &ls, int which, int32_t *idx, double *vals) {
  int64_t n = 0;
  for (size_t i = 0; i < ls.keys.size(); ++i) {
    if (which == 0 && !vlso::isDefined(ls.vals[i])) continue;
    if (idx) {
      int64_t c[D];
      vlso::decode<D>(ls.keys[i], c);
      for (int d = 0; d < D; ++d) idx[n * D + d] = int32_t(c[d]);
    }
    if (vals) vals[n] = ls.vals[i];
    ++n;
  }
  return n;
}

// MarkVoidPoints markers (default options) of the defined points, in the
// order of vlso_ls_get(which = 0).
template <int D> int64_t listVoidMarkers(vlso::LS<D> &ls, uint8_t *out) {
  const std::vector<uint8_t> m = vlso::voidMarkers<D>(ls);
  int64_t n = 0;
  for (size_t i = 0; i < ls.keys.size(); ++i) {
    if (!vlso::isDefined(ls.vals[i])) continue;
    if (out) out[n] = m[i];
    ++n;
  }
  return n;
}

// Point data of the defined points (vlso_ls_get order); -1 when the level
// set carries none.
template <int D>
int64_t listPointData(vlso::LS<D> &ls, int64_t *src, double *vel, double *diss) {
  if (ls.pd.empty()) return -1;
  int64_t n = 0;
  for (size_t i = 0; i < ls.keys.size(); ++i) {
    if (!vlso::isDefined(ls.vals[i])) continue;
    if (src) src[n] = ls.pd[i].src, vel[n] = ls.pd[i].vel, diss[n] = ls.pd[i].diss;
    ++n;
  }
  return n;
}

// Sharding settings of the next advections (vlso_set_shard).
bool g_ownZ = false;
int64_t g_ownLo = 0, g_ownHi = 0;
vlsg_reduce_cb g_reduceCb = nullptr;
void *g_reduceUser = nullptr;

vlso::Params toParams(const vlsg_advect_params *p) {
  vlso::Params P;
  P.spatial = p->spatial_scheme;
  P.temporal = p->temporal_scheme;
  P.timeStepRatio = p->time_step_ratio;
  P.dissipationAlpha = p->dissipation_alpha;
  P.advectionTime = p->advection_time;
  P.singleStep = p->single_step != 0;
  P.calculateNormalVectors = p->calculate_normal_vectors != 0;
  P.adaptiveTimeStepping = p->adaptive_time_stepping != 0;
  P.ignoreVoids = p->ignore_voids != 0;
  P.adaptiveSubdivisions = p->adaptive_subdivisions < 1 ? 1 : p->adaptive_subdivisions;
  P.checkDissipation = p->check_dissipation != 0;
  P.saveAdvectionVelocities = p->save_advection_velocities != 0;
  P.updatePointData = p->update_point_data != 0;
  P.trackPointData = p->track_point_data != 0;
  P.maxSteps = p->max_steps ? p->max_steps : 10000000u;
  if (p->max_dissipation > 0) P.maxDissipation = p->max_dissipation;
  return P;
}

template <int D>
int advectD(Handle **hs, int n, const vlsg_advect_params *p,
            const vlso::VelSource &v, vlsg_advect_result *r,
            vlsg_update_cb upd = nullptr, void *updUser = nullptr) {
  std::vector<vlso::LS<D>> lss;
  lss.reserve(n);
  for (int i = 0; i < n; ++i) lss.push_back(get<D>(hs[i]));
  vlso::Advector<D> adv(lss, toParams(p), v);
  adv.updateCb = upd;
  adv.updateUser = updUser;
  adv.ownZ = g_ownZ;
  adv.ownLo = g_ownLo;
  adv.ownHi = g_ownHi;
  adv.reduceCb = g_reduceCb;
  adv.reduceUser = g_reduceUser;
  adv.apply(*r);
  for (int i = 0; i < n; ++i) get<D>(hs[i]) = lss[i];
  return 0;
}
} // namespace

extern "C" {

const char *vlso_last_error() { return g_err.c_str(); }
void vlso_set_threads(int n) { omp_set_num_threads(n > 0 ? n : 1); }
int vlso_get_threads() { return omp_get_max_threads(); }

void *vlso_ls_new(int D, const int64_t *gmin, const int64_t *gmax,
                  const int32_t *bc, double delta) {
  auto *h = new Handle();
  h->D = D;
  if (D == 2) {
    h->l2.reset(new vlso::LS<2>());
    for (int d = 0; d < 2; ++d)
      h->l2->grid.minI[d] = gmin[d], h->l2->grid.maxI[d] = gmax[d], h->l2->grid.bc[d] = bc[d];
    h->l2->grid.delta = delta;
  } else {
    h->l3.reset(new vlso::LS<3>());
    for (int d = 0; d < 3; ++d)
      h->l3->grid.minI[d] = gmin[d], h->l3->grid.maxI[d] = gmax[d], h->l3->grid.bc[d] = bc[d];
    h->l3->grid.delta = delta;
  }
  return h;
}
void vlso_ls_free(void *p) { delete static_cast<Handle *>(p); }

void *vlso_ls_copy(void *p) {
  auto *h = static_cast<Handle *>(p);
  auto *c = new Handle();
  c->D = h->D;
  if (h->D == 2) c->l2.reset(new vlso::LS<2>(*h->l2));
  else c->l3.reset(new vlso::LS<3>(*h->l3));
  return c;
}

int vlso_ls_set(void *p, int64_t n, const int32_t *idx, const double *vals,
                int64_t nRuns, const int32_t *runStart, const int8_t *runSign,
                int width) {
  auto *h = static_cast<Handle *>(p);
  return guarded([&] {
    if (h->D == 2) {
      auto g = h->l2->grid;
      vlso::fromPoints<2>(*h->l2, g, n, idx, vals, nRuns, runStart, runSign, width);
    } else {
      auto g = h->l3->grid;
      vlso::fromPoints<3>(*h->l3, g, n, idx, vals, nRuns, runStart, runSign, width);
    }
    return 0;
  });
}

// which: 0 = defined points, 1 = whole map (defined + shell)
int64_t vlso_ls_get(void *p, int which, int32_t *idx, double *vals) {
  auto *h = static_cast<Handle *>(p);
  return h->D == 2 ? listPoints<2>(*h->l2, which, idx, vals)
                   : listPoints<3>(*h->l3, which, idx, vals);
}
// Owned z-slab (axis 2; axis -1 owns everything) and reduction callback of
// the following advections, as vlsg_set_owned_region /
// vlsg_set_reduction_callback set them for a context.
void vlso_set_shard(int axis, int64_t lo, int64_t hi, vlsg_reduce_cb cb, void *user) {
  g_ownZ = axis == 2;
  g_ownLo = lo;
  g_ownHi = hi;
  g_reduceCb = cb;
  g_reduceUser = user;
}

int64_t vlso_point_data(void *p, int64_t *src, double *vel, double *diss) {
  auto *h = static_cast<Handle *>(p);
  return h->D == 2 ? listPointData<2>(*h->l2, src, vel, diss)
                   : listPointData<3>(*h->l3, src, vel, diss);
}
int64_t vlso_void_markers(void *p, uint8_t *out) {
  auto *h = static_cast<Handle *>(p);
  return h->D == 2 ? listVoidMarkers<2>(*h->l2, out) : listVoidMarkers<3>(*h->l3, out);
}
int vlso_ls_width(void *p) {
  auto *h = static_cast<Handle *>(p);
  return h->D == 2 ? h->l2->width : h->l3->width;
}
void vlso_ls_set_width(void *p, int w) {
  auto *h = static_cast<Handle *>(p);
  if (h->D == 2) h->l2->width = w;
  else h->l3->width = w;
}
int64_t vlso_ls_far_queries(void *p) {
  auto *h = static_cast<Handle *>(p);
  return h->D == 2 ? h->l2->farQueries.load() : h->l3->farQueries.load();
}
// Value of arbitrary grid points (map value or the sign sentinel).
int vlso_ls_values_at(void *p, int64_t n, const int32_t *idx, double *out) {
  auto *h = static_cast<Handle *>(p);
  return guarded([&] {
    for (int64_t i = 0; i < n; ++i) {
      if (h->D == 2) {
        int64_t c[2] = {h->l2->grid.mapCoord(0, idx[2 * i]), h->l2->grid.mapCoord(1, idx[2 * i + 1])};
        out[i] = h->l2->at(vlso::encode<2>(c));
      } else {
        int64_t c[3];
        for (int d = 0; d < 3; ++d) c[d] = h->l3->grid.mapCoord(d, idx[3 * i + d]);
        out[i] = h->l3->at(vlso::encode<3>(c));
      }
    }
    return 0;
  });
}

int vlso_expand(void *p, int width) {
  auto *h = static_cast<Handle *>(p);
  return guarded([&] {
    if (h->D == 2) vlso::expand<2>(*h->l2, width);
    else vlso::expand<3>(*h->l3, width);
    return 0;
  });
}
int vlso_reduce(void *p, int width) {
  auto *h = static_cast<Handle *>(p);
  return guarded([&] {
    if (h->D == 2) vlso::reduce<2>(*h->l2, width);
    else vlso::reduce<3>(*h->l3, width);
    return 0;
  });
}
int vlso_prune(void *p, int removeStrayZeros) {
  auto *h = static_cast<Handle *>(p);
  return guarded([&] {
    if (h->D == 2) vlso::prune<2>(*h->l2, removeStrayZeros != 0);
    else vlso::prune<3>(*h->l3, removeStrayZeros != 0);
    return 0;
  });
}
int vlso_rebuild(void *p, double cutoff, int finalWidth) {
  auto *h = static_cast<Handle *>(p);
  return guarded([&] {
    if (h->D == 2) vlso::rebuild<2>(*h->l2, cutoff, finalWidth);
    else vlso::rebuild<3>(*h->l3, cutoff, finalWidth);
    return 0;
  });
}
// op: 0 INTERSECT, 1 UNION, 2 RELATIVE_COMPLEMENT (lsBooleanOperation.hpp:27-33)
int vlso_boolean(void *a, void *b, int op) {
  auto *A = static_cast<Handle *>(a);
  auto *B = static_cast<Handle *>(b);
  return guarded([&] {
    auto run = [&](auto &la, auto &lb) {
      if (op == 0) vlso::booleanOp(la, lb, vlso::maxComp);
      else if (op == 1) vlso::booleanOp(la, lb, vlso::minComp);
      else if (op == 2)
        vlso::booleanOp(la, lb, [](double x, double y) { return vlso::maxComp(x, -y); });
      else throw std::runtime_error("boolean op not supported");
    };
    if (A->D == 2) run(*A->l2, *B->l2);
    else run(*A->l3, *B->l3);
    return 0;
  });
}
int64_t vlso_check(void *p) {
  auto *h = static_cast<Handle *>(p);
  return h->D == 2 ? vlso::check<2>(*h->l2) : vlso::check<3>(*h->l3);
}
int vlso_chamfer(void *t, void *s, double *out, int64_t *counts) {
  auto *T = static_cast<Handle *>(t);
  auto *S = static_cast<Handle *>(s);
  return guarded([&] {
    if (T->D == 2) vlso::chamfer<2>(*T->l2, *S->l2, out, counts);
    else vlso::chamfer<3>(*T->l3, *S->l3, out, counts);
    return 0;
  });
}
int64_t vlso_surface_nodes(void *p, double *out, int64_t cap) {
  auto *h = static_cast<Handle *>(p);
  std::vector<double> nodes = h->D == 2 ? vlso::surfaceNodes<2>(*h->l2)
                                        : vlso::surfaceNodes<3>(*h->l3);
  const int64_t n = nodes.size() / h->D;
  if (out)
    for (int64_t i = 0; i < std::min(n, cap) * h->D; ++i) out[i] = nodes[i];
  return n;
}

int vlso_advect(void **lss, int n, const vlsg_advect_params *p,
                const vlsg_velocity_desc *v, vlsg_advect_result *r) {
  auto **hs = reinterpret_cast<Handle **>(lss);
  return guarded([&] {
    if (n < 1) throw std::runtime_error("no level sets");
    vlso::VelSource vs;
    vs.desc = *v;
    return hs[0]->D == 2 ? advectD<2>(hs, n, p, vs, r) : advectD<3>(hs, n, p, vs, r);
  });
}

// The same with a host velocity callback (called one point at a time, from
// the OpenMP threads).
int vlso_advect_cb(void **lss, int n, const vlsg_advect_params *p, vlsg_velocity_cb cb,
                   void *user, vlsg_alpha_cb alphaCb, void *alphaUser, vlsg_advect_result *r) {
  auto **hs = reinterpret_cast<Handle **>(lss);
  return guarded([&] {
    if (n < 1) throw std::runtime_error("no level sets");
    if (!cb) throw std::runtime_error("no velocity callback");
    vlso::VelSource vs;
    vs.cb = cb;
    vs.user = user;
    vs.alphaCb = alphaCb;
    vs.alphaUser = alphaUser;
    return hs[0]->D == 2 ? advectD<2>(hs, n, p, vs, r) : advectD<3>(hs, n, p, vs, r);
  });
}

// Either velocity form (desc when cb is NULL) with a velocity-update callback.
int vlso_advect_ex(void **lss, int n, const vlsg_advect_params *p, const vlsg_velocity_desc *desc,
                   vlsg_velocity_cb cb, void *user, vlsg_alpha_cb alphaCb, void *alphaUser,
                   vlsg_update_cb upd, void *updUser, vlsg_advect_result *r) {
  auto **hs = reinterpret_cast<Handle **>(lss);
  return guarded([&] {
    if (n < 1) throw std::runtime_error("no level sets");
    vlso::VelSource vs;
    if (cb) {
      vs.cb = cb;
      vs.user = user;
      vs.alphaCb = alphaCb;
      vs.alphaUser = alphaUser;
    } else {
      if (!desc) throw std::runtime_error("no velocity");
      vs.desc = *desc;
    }
    return hs[0]->D == 2 ? advectD<2>(hs, n, p, vs, r, upd, updUser)
                         : advectD<3>(hs, n, p, vs, r, upd, updUser);
  });
}

// Prepare / FinalizeStencilLocalLaxFriedrichs on level sets bottom..top.
int vlso_prepare_stencil_llf(void **lss, int n, const int32_t *isDepo, int nd) {
  auto **hs = reinterpret_cast<Handle **>(lss);
  return guarded([&] {
    if (n < 1) throw std::runtime_error("no level sets");
    std::vector<bool> depo(nd);
    for (int i = 0; i < nd; ++i) depo[i] = isDepo[i] != 0;
    auto run = [&](auto dim) {
      constexpr int D = decltype(dim)::value;
      std::vector<vlso::LS<D>> v;
      for (int i = 0; i < n; ++i) v.push_back(get<D>(hs[i]));
      vlso::prepareStencilLLF<D>(v, depo);
      get<D>(hs[n - 1]) = v.back();
    };
    if (hs[0]->D == 2) run(std::integral_constant<int, 2>());
    else run(std::integral_constant<int, 3>());
    return 0;
  });
}
int vlso_finalize_stencil_llf(void **lss, int n) {
  auto **hs = reinterpret_cast<Handle **>(lss);
  return guarded([&] {
    if (n < 2) throw std::runtime_error("FinalizeStencilLocalLaxFriedrichs needs two level sets");
    auto run = [&](auto dim) {
      constexpr int D = decltype(dim)::value;
      std::vector<vlso::LS<D>> v;
      for (int i = 0; i < n; ++i) v.push_back(get<D>(hs[i]));
      vlso::finalizeStencilLLF<D>(v);
      get<D>(hs[n - 1]) = v.back();
    };
    if (hs[0]->D == 2) run(std::integral_constant<int, 2>());
    else run(std::integral_constant<int, 3>());
    return 0;
  });
}

} // extern "C"
