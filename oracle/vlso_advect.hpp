// vlso_advect.hpp -- TEST INFRASTRUCTURE ONLY (the oracle): FP64 restatement
// of viennals::Advect<double,D> (lsAdvect.hpp), its spatial schemes
// (lsEngquistOsher.hpp, lsLaxFriedrichs.hpp, lsLocalLaxFriedrichs.hpp,
// lsLocalLocalLaxFriedrichs.hpp, lsWENO.hpp + lsFiniteDifferences.hpp) and
// time integration (lsAdvectIntegrationSchemes.hpp).  Build with
// -ffp-contract=off: every expression keeps the reference's evaluation order.
//
// One deliberate choice: the reference accumulates the Lax-Friedrichs
// dissipation coefficients of LocalLaxFriedrichs / LocalLocalLaxFriedrichs per
// OpenMP thread and bounds the time step per thread (lsAdvect.hpp:493,
// :595-606), which makes dt depend on the thread count.  Here the maximum is
// taken over all points, i.e. the reference run with one thread.
#pragma once

#include <cfloat>

#include "vlso_core.hpp"

namespace vlso {

inline double pow2(double v) { return v * v; }
inline double stdMax(double a, double b) { return (a < b) ? b : a; }
inline double stdMin(double a, double b) { return (b < a) ? b : a; }

// Velocity functor of vlsg.h (vlsg_velocity_desc), evaluated term by term.
inline double scalarVelocity(const vlsg_velocity_desc &v, int material,
                             const double n[3]) {
  int m = material < v.n_materials ? material : v.n_materials - 1;
  if (m < 0) m = 0;
  double s = v.rate[m];
  for (int k = 0; k < 3; ++k) {
    const double c = n[k] > 0 ? v.lin_pos[m][k] : v.lin_neg[m][k];
    if (c != 0) s = s + c * n[k];
  }
  for (int k = 0; k < 3; ++k) {
    const double c = n[k] > 0 ? v.abs_pos[m][k] : v.abs_neg[m][k];
    if (c != 0) s = s + c * std::fabs(n[k]);
  }
  for (int k = 0; k < 3; ++k) {
    const double c = n[k] > 0 ? v.sq_pos[m][k] : v.sq_neg[m][k];
    if (c != 0) s = s + c * (n[k] * n[k]);
  }
  return s;
}
inline void vectorVelocity(const vlsg_velocity_desc &v, int material,
                           double out[3]) {
  int m = material < v.n_materials ? material : v.n_materials - 1;
  if (m < 0) m = 0;
  for (int k = 0; k < 3; ++k) out[k] = v.vec[m][k];
}

// The velocity of one evaluation: the functor of vlsg.h, or a host callback
// (VelocityField::getScalarVelocity and getVectorVelocity,
// lsVelocityField.hpp:17-30) asked one point at a time with the coordinate
// (index * gridDelta), the material, the normal and the point id the
// reference passes.  A callback failure is recorded and reported after the
// parallel loop that met it.
struct VelSource {
  vlsg_velocity_desc desc{};
  vlsg_velocity_cb cb = nullptr;
  void *user = nullptr;
  mutable std::atomic<int> failed{0};
  VelSource() = default;
  VelSource(const VelSource &o)
      : desc(o.desc), cb(o.cb), user(o.user), alphaCb(o.alphaCb), alphaUser(o.alphaUser) {}
  void query(const double coord[3], int material, const double n[3], uint64_t pointId,
             double &scalar, double vec[3]) const {
    if (!cb) {
      scalar = scalarVelocity(desc, material, n);
      vectorVelocity(desc, material, vec);
      return;
    }
    const int32_t m = material;
    if (cb(user, 1, coord, &m, n, &pointId, &scalar, vec) != 0) {
      failed = 1;
      scalar = 0;
      vec[0] = vec[1] = vec[2] = 0;
    }
  }
  vlsg_alpha_cb alphaCb = nullptr;
  void *alphaUser = nullptr;
  // getDissipationAlpha(direction, material, centralDifferences)
  double alpha(int dir, int material, const double cd[3]) const {
    if (!cb) {
      int m = material < desc.n_materials ? material : desc.n_materials - 1;
      if (m < 0) m = 0;
      return desc.alpha[m][dir];
    }
    if (!alphaCb) return 0.;
    const int32_t d = dir, m = material;
    double a = 0;
    if (alphaCb(alphaUser, 1, &d, &m, cd, &a) != 0) failed = 1;
    return a;
  }
  void check() const {
    if (failed) throw std::runtime_error("the velocity callback failed");
  }
};

// Point id of every map entry: its rank among the defined points in HRLE
// order (the id viennahrle's iterators report, lsAdvect.hpp:169).
template <int D> std::vector<uint64_t> pointIds(const LS<D> &t) {
  std::vector<uint64_t> id(t.keys.size());
  uint64_t k = 0;
  for (size_t i = 0; i < t.keys.size(); ++i) {
    id[i] = k;
    if (isDefined(t.vals[i])) ++k;
  }
  return id;
}

template <int D> void coordinateOf(const Grid<D> &g, uint64_t key, double c[3]) {
  c[0] = c[1] = c[2] = 0.;
  for (int d = 0; d < D; ++d) c[d] = double(coordOf<D>(key, d)) * g.delta;
}

struct Params {
  int spatial = VLSG_ENGQUIST_OSHER_1ST_ORDER;
  int temporal = VLSG_FORWARD_EULER;
  double timeStepRatio = 0.4999;
  double dissipationAlpha = 1.0;
  double advectionTime = 0.;
  bool singleStep = false;
  bool calculateNormalVectors = true;
  bool adaptiveTimeStepping = false;
  bool ignoreVoids = false; // setIgnoreVoids, lsAdvect.hpp:899
  unsigned adaptiveSubdivisions = 20;
  bool checkDissipation = true;
  bool saveAdvectionVelocities = false; // lsAdvect.hpp:916
  bool updatePointData = true;          // lsAdvect.hpp:962
  bool trackPointData = false;          // carry point data through apply
  uint32_t maxSteps = 10000000;
  // StencilLocalLaxFriedrichsScalar::setMaxDissipation (static, default max)
  double maxDissipation = std::numeric_limits<double>::max();
  // baseNormalEpsilon of StencilLocalLaxFriedrichsScalar (:44-45)
  double baseNormalEpsilon = std::cbrt(std::numeric_limits<double>::epsilon());
  static constexpr double integrationCutoff = 0.5;    // lsAdvect.hpp:77
  static constexpr double wrappingLayerEpsilon = 1e-4; // lsAdvect.hpp:80
};

// Expand width each scheme's prepareLS asks for.
inline int schemeWidth(int s) {
  switch (s) {
  case VLSG_ENGQUIST_OSHER_1ST_ORDER: return 3;          // lsEngquistOsher.hpp:31
  case VLSG_ENGQUIST_OSHER_2ND_ORDER: return 5;
  case VLSG_LAX_FRIEDRICHS_1ST_ORDER: return 3;          // lsLaxFriedrichs.hpp:225
  case VLSG_LAX_FRIEDRICHS_2ND_ORDER: return 5;
  case VLSG_LOCAL_LOCAL_LAX_FRIEDRICHS_1ST_ORDER: return 3; // lsLocalLocalLaxFriedrichs.hpp:288
  case VLSG_LOCAL_LOCAL_LAX_FRIEDRICHS_2ND_ORDER: return 5;
  case VLSG_LOCAL_LAX_FRIEDRICHS_1ST_ORDER: return 7;    // lsLocalLaxFriedrichs.hpp:55
  case VLSG_LOCAL_LAX_FRIEDRICHS_2ND_ORDER: return 9;
  case VLSG_LOCAL_LAX_FRIEDRICHS_ANALYTICAL_1ST_ORDER: return 7; // lsLocalLaxFriedrichsAnalytical.hpp:52
  case VLSG_STENCIL_LOCAL_LAX_FRIEDRICHS_1ST_ORDER: return 8; // lsStencilLocalLaxFriedrichsScalar.hpp:207
  case VLSG_WENO_3RD_ORDER: return 5;                    // lsWENO.hpp:44 (r=2)
  case VLSG_WENO_5TH_ORDER: return 7;                    // (r=3)
  default: return -1;
  }
}
inline bool schemeSupported(int s) { return schemeWidth(s) > 0; }

// Central/one-sided differences with the second-order correction of
// lsEngquistOsher.hpp:59-111 (identical in lsLaxFriedrichs.hpp:256-309,
// lsLocalLaxFriedrichs.hpp:85-143, lsLocalLocalLaxFriedrichs.hpp:318-371).
template <int D, class F>
inline void oneSided(F V, int i, double phi0, double gridDelta, int order,
                     double &diffPos, double &diffNeg) {
  const double deltaPos = gridDelta;
  const double deltaNeg = -gridDelta;
  const double phiPos = V(i, 1);
  const double phiNeg = V(i, -1);
  diffPos = (phiPos - phi0) / deltaPos;
  diffNeg = (phiNeg - phi0) / deltaNeg;
  if (order == 2) {
    const double deltaPosPos = 2 * gridDelta;
    const double deltaNegNeg = -2 * gridDelta;
    const double phiPosPos = V(i, 2);
    const double phiNegNeg = V(i, -2);
    const double diff00 =
        (((deltaNeg * phiPos - deltaPos * phiNeg) / (deltaPos - deltaNeg) +
          phi0)) /
        (deltaPos * deltaNeg);
    const double diffNegNeg = (((deltaNeg * phiNegNeg - deltaNegNeg * phiNeg) /
                                    (deltaNegNeg - deltaNeg) +
                                phi0)) /
                              (deltaNegNeg * deltaNeg);
    const double diffPosPos = (((deltaPos * phiPosPos - deltaPosPos * phiPos) /
                                    (deltaPosPos - deltaPos) +
                                phi0)) /
                              (deltaPosPos * deltaPos);
    if (std::signbit(diff00) == std::signbit(diffPosPos)) {
      if (std::abs(diffPosPos * deltaPos) < std::abs(diff00 * deltaNeg))
        diffPos -= deltaPos * diffPosPos;
      else
        diffPos += deltaNeg * diff00;
    }
    if (std::signbit(diff00) == std::signbit(diffNegNeg)) {
      if (std::abs(diffNegNeg * deltaNeg) < std::abs(diff00 * deltaPos))
        diffNeg -= deltaNeg * diffNegNeg;
      else
        diffNeg += deltaPos * diff00;
    }
  }
}

// FiniteDifferences::weno3 / weno5, lsFiniteDifferences.hpp:58-123.
inline double weno3(const double *x, double delta, bool plus,
                    double eps = 1e-6) {
  double d[3];
  if (plus) {
    d[0] = x[2] - x[1];
    d[1] = x[3] - x[2];
    d[2] = x[4] - x[3];
    double N = eps + pow2(d[2] - d[1]);
    double Dd = eps + pow2(d[1] - d[0]);
    double D2 = Dd * Dd;
    double wp = D2 / (D2 + 2 * N * N);
    return (d[0] + d[1] - wp * (d[2] - 2 * d[1] + d[0])) / (2 * delta);
  }
  d[0] = x[1] - x[0];
  d[1] = x[2] - x[1];
  d[2] = x[3] - x[2];
  double N = eps + pow2(d[1] - d[0]);
  double Dd = eps + pow2(d[2] - d[1]);
  double D2 = Dd * Dd;
  double wp = D2 / (D2 + 2 * N * N);
  return (d[1] + d[2] - wp * (d[0] - 2 * d[1] + d[2])) / (2 * delta);
}
inline double weno5(const double *x, double dx, bool plus, double eps = 1e-6) {
  double d[5];
  if (!plus) {
    for (int i = 0; i < 5; ++i) d[i] = x[i + 1] - x[i];
  } else {
    for (int i = 0; i < 5; ++i) d[i] = x[6 - i] - x[5 - i];
  }
  double s1 = double(13.0 / 12.0) * pow2(d[0] - 2 * d[1] + d[2]) +
              double(1.0 / 4.0) * pow2(d[0] - 4 * d[1] + 3 * d[2]);
  double s2 = double(13.0 / 12.0) * pow2(d[1] - 2 * d[2] + d[3]) +
              double(1.0 / 4.0) * pow2(d[1] - d[3]);
  double s3 = double(13.0 / 12.0) * pow2(d[2] - 2 * d[3] + d[4]) +
              double(1.0 / 4.0) * pow2(3 * d[2] - 4 * d[3] + d[4]);
  double eps_scaled = eps * dx * dx;
  double al1 = double(0.1) / (eps_scaled + s1);
  double al2 = double(0.6) / (eps_scaled + s2);
  double al3 = double(0.3) / (eps_scaled + s3);
  double alsum = al1 + al2 + al3;
  double p1 = double(1.0 / 6.0) * (2 * d[0] - 7 * d[1] + 11 * d[2]);
  double p2 = double(1.0 / 6.0) * (-d[1] + 5 * d[2] + 2 * d[3]);
  double p3 = double(1.0 / 6.0) * (2 * d[2] + 5 * d[3] - d[4]);
  return (al1 * p1 + al2 * p2 + al3 * p3) / (alsum * dx);
}

template <int D> struct SchemeCtx {
  const LS<D> &top;
  const Params &P;
  const VelSource &vel;
  const double *globalAlphas; // LF: findGlobalAlphas result
};

// One scheme evaluation at `key` for `material` (operator() of each scheme).
// `alphas` accumulates finalAlphas of LLF / LLLF.
template <int D>
std::pair<double, double> evalScheme(const SchemeCtx<D> &S, uint64_t key,
                                     uint64_t pointId, int material, double *alphas) {
  const LS<D> &ls = S.top;
  const Grid<D> &g = ls.grid;
  const double gridDelta = g.delta;
  const int sch = S.P.spatial;
  auto V = [&](int d, int off) { return ls.at(shiftKey<D>(g, key, d, off)); };
  const double C = ls.at(key);
  double coordinate[3];
  coordinateOf<D>(g, key, coordinate);

  if (sch == VLSG_STENCIL_LOCAL_LAX_FRIEDRICHS_1ST_ORDER) {
    // StencilLocalLaxFriedrichsScalar<T,D,1> with FIRST_ORDER differences and
    // ADAPTIVE_EPSILON_STRATEGY 1 (lsStencilLocalLaxFriedrichsScalar.hpp:219-400).
    // `alphas` receives this call's finalAlphas and alphas[3] = 1 when the
    // call gets past the zero-velocity return (they bound the time step).
    auto VI = [&](const int *off) { return ls.at(offsetKey<D>(g, key, off)); };
    // component i of calculateGradient / calculateNormal at `off`: the three
    // values along i are taken with coordinate i set to -1, 0, 1 (:342-352,
    // :360-372), whatever off[i] is
    auto grad1 = [&](const int *off, int i) {
      int o[D];
      for (int d = 0; d < D; ++d) o[d] = off[d];
      double v[3];
      for (int j = 0; j < 3; ++j) {
        o[i] = j - 1;
        v[j] = VI(o);
      }
      const double dNeg = (v[1] - v[0]) / gridDelta; // lsFiniteDifferences.hpp:132-134
      const double dPos = (v[2] - v[1]) / gridDelta; // :155-157
      return (dPos + dNeg) * 0.5;                    // :177-181
    };
    auto normalAt = [&](const int *off, double *n) {
      n[0] = n[1] = n[2] = 0.;
      double modulus = 0.;
      for (int i = 0; i < D; ++i) {
        n[i] = grad1(off, i);
        modulus += n[i] * n[i];
      }
      modulus = 1. / std::sqrt(modulus);
      for (int i = 0; i < D; ++i) n[i] *= modulus;
    };
    int zero[D];
    for (int d = 0; d < D; ++d) zero[d] = 0;
    double normalVector[3];
    normalAt(zero, normalVector);
    double scalarVelocity, vectorVelocity[3];
    S.vel.query(coordinate, material, normalVector, pointId, scalarVelocity, vectorVelocity);
    for (int i = 0; i < D; ++i) scalarVelocity += vectorVelocity[i] * normalVector[i];
    if (scalarVelocity == 0.) return {0, 0};
    double gradSq = 0.; // Norm(calculateGradient(0))
    for (int i = 0; i < D; ++i) {
      const double gi = grad1(zero, i);
      gradSq += gi * gi;
    }
    const double hamiltonian = std::sqrt(gradSq) * scalarVelocity;
    constexpr int numStencil = D == 3 ? 27 : 9;
    double sa[27][3] = {};
    int cur[D];
    for (int d = 0; d < D; ++d) cur[d] = -1;
    for (int st = 0; st < numStencil; ++st) {
      double localNormal[3];
      normalAt(cur, localNormal);
      // a corrupted normal leaves the stencil index where it is (:288-293)
      if (std::abs(localNormal[0]) < 1e-6 && std::abs(localNormal[1]) < 1e-6 &&
          std::abs(localNormal[2]) < 1e-6)
        continue;
      double localCoord[3] = {coordinate[0], coordinate[1], coordinate[2]};
      for (int dir = 0; dir < D; ++dir) localCoord[dir] += cur[dir] * gridDelta;
      double lsv, lvv[3];
      S.vel.query(localCoord, material, localNormal, pointId, lsv, lvv);
      for (int dir = 0; dir < D; ++dir) lsv += lvv[dir] * localNormal[dir];
      // calculateSimpleAdaptiveEpsilon, :60-75
      const double absVel = std::abs(lsv);
      const double baseEps = S.P.baseNormalEpsilon * gridDelta;
      double DN = baseEps;
      if (absVel > 1e-10) {
        const double scale = stdMax(0.1, stdMin(10.0, absVel));
        DN = baseEps * scale;
      }
      double np[3] = {localNormal[0], localNormal[1], localNormal[2]};
      double nn[3] = {localNormal[0], localNormal[1], localNormal[2]};
      double velocityDelta[3] = {0, 0, 0};
      for (int k = 0; k < D; ++k) {
        np[k] -= DN;
        nn[k] += DN;
        double vp, vn, unused[3];
        S.vel.query(localCoord, material, np, pointId, vp, unused);
        S.vel.query(localCoord, material, nn, pointId, vn, unused);
        velocityDelta[k] = (vn - vp) / (2.0 * DN);
        np[k] += DN;
        nn[k] -= DN;
      }
      for (int k = 0; k < D; ++k) {
        double gradient[3];
        for (int i = 0; i < D; ++i) gradient[i] = grad1(cur, i);
        double monti = 0, toifl = 0;
        for (int j = 0; j < D - 1; ++j) {
          const int idx = (k + 1 + j) % D;
          monti += gradient[idx] * gradient[idx];
          toifl += gradient[idx] * velocityDelta[idx];
        }
        double denom = 0;
        for (int i = 0; i < D; ++i) denom += gradient[i] * gradient[i];
        monti *= velocityDelta[k] / denom;
        toifl *= -gradient[k] / denom;
        const double osher = lsv * localNormal[k];
        sa[st][k] = std::fabs(monti + toifl + osher);
      }
      // incrementIndex, :196-204
      int dim = 0;
      for (; dim < D - 1; ++dim) {
        if (cur[dim] < 1) break;
        cur[dim] = -1;
      }
      ++cur[dim];
    }
    double dissipation = 0.;
    for (int d = 0; d < D; ++d) {
      int o[D];
      for (int e = 0; e < D; ++e) o[e] = 0;
      double v[3];
      for (int j = 0; j < 3; ++j) {
        o[d] = j - 1;
        v[j] = VI(o);
      }
      const double dNeg = (v[1] - v[0]) / gridDelta;
      const double dPos = (v[2] - v[1]) / gridDelta;
      const double gradientDiff = (dPos - dNeg) * 0.5; // :183-187
      double maxAlpha = 0;
      for (int i = 0; i < numStencil; ++i) maxAlpha = stdMax(maxAlpha, sa[i][d]);
      const double finalAlpha = stdMin(maxAlpha, S.P.maxDissipation);
      alphas[d] = finalAlpha;
      dissipation += finalAlpha * gradientDiff;
    }
    alphas[3] = 1.;
    return {hamiltonian, dissipation};
  }

  if (sch == VLSG_WENO_3RD_ORDER || sch == VLSG_WENO_5TH_ORDER) {
    // lsWENO.hpp:53-160
    const int r = sch == VLSG_WENO_3RD_ORDER ? 2 : 3;
    double gradPosTotal = 0, gradNegTotal = 0;
    double wMinus[D], wPlus[D], st[7];
    for (int i = 0; i < D; i++) {
      st[r] = C;
      for (int k = 1; k <= r; ++k) {
        st[r + k] = V(i, k);
        st[r - k] = V(i, -k);
      }
      if (r == 2) {
        wMinus[i] = weno3(st, gridDelta, false);
        wPlus[i] = weno3(st, gridDelta, true);
      } else {
        wMinus[i] = weno5(st, gridDelta, false);
        wPlus[i] = weno5(st, gridDelta, true);
      }
      gradPosTotal += pow2(stdMax(wMinus[i], 0.)) + pow2(stdMin(wPlus[i], 0.));
      gradNegTotal += pow2(stdMin(wMinus[i], 0.)) + pow2(stdMax(wPlus[i], 0.));
    }
    double vel_grad = 0.;
    double n[3] = {0, 0, 0};
    // Advect passes dissipationAlpha as the calcNormal flag (lsAdvect.hpp:670-676)
    if (S.P.dissipationAlpha != 0.0) {
      double denominator = 0;
      for (int i = 0; i < D; i++) {
        const double pos = V(i, 1);
        const double neg = V(i, -1);
        n[i] = pos - neg;
        denominator += n[i] * n[i];
      }
      if (denominator > 0) {
        denominator = 1. / std::sqrt(denominator);
        for (int i = 0; i < D; ++i) n[i] *= denominator;
      }
    }
    double scalarVel, vv[3];
    S.vel.query(coordinate, material, n, pointId, scalarVel, vv);
    if (scalarVel > 0)
      vel_grad += std::sqrt(gradPosTotal) * scalarVel;
    else
      vel_grad += std::sqrt(gradNegTotal) * scalarVel;
    for (int w = 0; w < D; w++) {
      if (vv[w] > 0.)
        vel_grad += vv[w] * wMinus[w];
      else
        vel_grad += vv[w] * wPlus[w];
    }
    return {vel_grad, 0.};
  }

  const int order = (sch == VLSG_ENGQUIST_OSHER_2ND_ORDER ||
                     sch == VLSG_LAX_FRIEDRICHS_2ND_ORDER ||
                     sch == VLSG_LOCAL_LOCAL_LAX_FRIEDRICHS_2ND_ORDER ||
                     sch == VLSG_LOCAL_LAX_FRIEDRICHS_2ND_ORDER)
                        ? 2
                        : 1;
  double gradPos[D], gradNeg[D];

  if (sch == VLSG_ENGQUIST_OSHER_1ST_ORDER ||
      sch == VLSG_ENGQUIST_OSHER_2ND_ORDER) {
    // lsEngquistOsher.hpp:42-162
    double gradPosTotal = 0, gradNegTotal = 0;
    for (int i = 0; i < D; i++) {
      double diffPos, diffNeg;
      oneSided<D>(V, i, C, gridDelta, order, diffPos, diffNeg);
      gradPos[i] = diffNeg;
      gradNeg[i] = diffPos;
      gradPosTotal += pow2(stdMax(diffNeg, 0.)) + pow2(stdMin(diffPos, 0.));
      gradNegTotal += pow2(stdMin(diffNeg, 0.)) + pow2(stdMax(diffPos, 0.));
    }
    double vel_grad = 0.;
    double n[3] = {0, 0, 0};
    if (S.P.calculateNormalVectors) {
      double denominator = 0;
      for (int i = 0; i < D; i++) {
        const double pos = V(i, 1) - C;
        const double neg = C - V(i, -1);
        n[i] = (pos + neg) * 0.5;
        denominator += n[i] * n[i];
      }
      denominator = 1. / std::sqrt(denominator);
      for (int i = 0; i < D; ++i) n[i] *= denominator;
    }
    double sv, vv[3];
    S.vel.query(coordinate, material, n, pointId, sv, vv);
    if (sv > 0)
      vel_grad += std::sqrt(gradPosTotal) * sv;
    else
      vel_grad += std::sqrt(gradNegTotal) * sv;
    for (int w = 0; w < D; w++) {
      if (vv[w] > 0.)
        vel_grad += vv[w] * gradPos[w];
      else
        vel_grad += vv[w] * gradNeg[w];
    }
    return {vel_grad, 0.};
  }

  // Lax-Friedrichs family: central gradient, dissipation from alphas.
  const bool globalLF = (sch == VLSG_LAX_FRIEDRICHS_1ST_ORDER ||
                         sch == VLSG_LAX_FRIEDRICHS_2ND_ORDER);
  const bool calcNormal = globalLF ? S.P.calculateNormalVectors : true;
  const double alphaFactor = S.P.dissipationAlpha;
  double grad = 0., dissipation = 0.;
  double n[3] = {0, 0, 0};
  double normalModulus = 0;
  for (int i = 0; i < D; i++) {
    double diffPos, diffNeg;
    oneSided<D>(V, i, C, gridDelta, order, diffPos, diffNeg);
    gradPos[i] = diffNeg;
    gradNeg[i] = diffPos;
    if (calcNormal) {
      n[i] = (diffNeg + diffPos) * 0.5;
      normalModulus += n[i] * n[i];
    }
    grad += pow2((diffNeg + diffPos) * 0.5);
    if (globalLF) // lsLaxFriedrichs.hpp:317
      dissipation +=
          alphaFactor * S.globalAlphas[i] * (diffPos - diffNeg) * 0.5;
  }
  if (calcNormal) {
    normalModulus = 1. / std::sqrt(normalModulus);
    for (int i = 0; i < D; ++i) n[i] *= normalModulus;
  }
  double sv, vv[3];
  S.vel.query(coordinate, material, n, pointId, sv, vv);
  double totalGrad = 0.;
  if (sv != 0.) totalGrad = sv * std::sqrt(grad);
  for (int w = 0; w < D; w++) {
    if (vv[w] > 0.)
      totalGrad += vv[w] * gradPos[w];
    else
      totalGrad += vv[w] * gradNeg[w];
  }
  if (globalLF) // lsLaxFriedrichs.hpp:347
    return {totalGrad, ((totalGrad != 0.) ? dissipation : 0)};

  if (totalGrad == 0.) return {0, 0}; // lsLocalLaxFriedrichs.hpp:179-181

  if (sch == VLSG_LOCAL_LAX_FRIEDRICHS_ANALYTICAL_1ST_ORDER) {
    // lsLocalLaxFriedrichsAnalytical.hpp:183-225: the user's alphas at the
    // 3^D box (central differences, not normalised), no alphaFactor
    double alpha[D];
    for (int i = 0; i < D; ++i) alpha[i] = 0;
    int nIdx[D];
    for (int d = 0; d < D; ++d) nIdx[d] = -1;
    int numNeighbors = 1;
    for (int d = 0; d < D; ++d) numNeighbors *= 3;
    auto VB = [&](const int *off) { return ls.at(offsetKey<D>(g, key, off)); };
    for (int q = 0; q < numNeighbors; ++q) {
      double normal[3] = {0, 0, 0};
      const double center = VB(nIdx);
      for (int dir = 0; dir < D; ++dir) {
        int o[D];
        for (int d = 0; d < D; ++d) o[d] = nIdx[d];
        o[dir] = nIdx[dir] - 1;
        const double neg = VB(o);
        o[dir] = nIdx[dir] + 1;
        const double pos = VB(o);
        // calculateNormalComponent, :30-34
        const double dPos = (pos - center) / gridDelta;
        const double dNeg = (center - neg) / gridDelta;
        normal[dir] = (dPos + dNeg) * 0.5;
      }
      for (int dir = 0; dir < D; ++dir) {
        const double tempAlpha = S.vel.alpha(dir, material, normal);
        alpha[dir] = stdMax(alpha[dir], tempAlpha);
        alphas[dir] = stdMax(alphas[dir], tempAlpha);
      }
      int dim = 0;
      for (; dim < D - 1; ++dim) {
        if (nIdx[dim] < 1) break;
        nIdx[dim] = -1;
      }
      ++nIdx[dim];
    }
    for (int i = 0; i < D; ++i) dissipation += alpha[i] * (gradNeg[i] - gradPos[i]) * 0.5;
    return {totalGrad, dissipation};
  }

  if (sch == VLSG_LOCAL_LOCAL_LAX_FRIEDRICHS_1ST_ORDER ||
      sch == VLSG_LOCAL_LOCAL_LAX_FRIEDRICHS_2ND_ORDER) {
    // lsLocalLocalLaxFriedrichs.hpp:413-420
    for (int i = 0; i < D; ++i) {
      const double alpha = std::abs((sv + vv[i]) * n[i]);
      alphas[i] = stdMax(alphas[i], alpha);
      dissipation += alphaFactor * alpha * (gradNeg[i] - gradPos[i]) * 0.5;
    }
    return {totalGrad, dissipation};
  }

  // LocalLaxFriedrichs: alphas over the 3^D box, lsLocalLaxFriedrichs.hpp:183-240
  double alpha[D];
  for (int i = 0; i < D; ++i) alpha[i] = 0;
  int nIdx[D];
  for (int d = 0; d < D; ++d) nIdx[d] = -1;
  int numNeighbors = 1;
  for (int d = 0; d < D; ++d) numNeighbors *= 3;
  auto VB = [&](const int *off) { return ls.at(offsetKey<D>(g, key, off)); };
  for (int q = 0; q < numNeighbors; ++q) {
    double normal[3] = {0, 0, 0};
    double nm = 0.;
    const double center = VB(nIdx);
    for (int dir = 0; dir < D; ++dir) {
      int o[D];
      for (int d = 0; d < D; ++d) o[d] = nIdx[d];
      o[dir] = nIdx[dir] - 1;
      const double neg = VB(o);
      o[dir] = nIdx[dir] + 1;
      const double pos = VB(o);
      // calculateNormalComponent, :32-36
      const double dPos = (pos - center) / gridDelta;
      const double dNeg = (center - neg) / gridDelta;
      normal[dir] = (dPos + dNeg) * 0.5;
      nm += normal[dir] * normal[dir];
    }
    nm = 1. / std::sqrt(nm);
    for (int dir = 0; dir < D; ++dir) normal[dir] *= nm;
    double coords[3] = {0, 0, 0};
    for (int dir = 0; dir < D; ++dir) coords[dir] = coordinate[dir] + nIdx[dir] * gridDelta;
    double scaVel, vecVel[3];
    S.vel.query(coords, material, normal, pointId, scaVel, vecVel);
    for (int dir = 0; dir < D; ++dir) {
      const double tempAlpha = std::abs((scaVel + vecVel[dir]) * normal[dir]);
      alpha[dir] = stdMax(alpha[dir], tempAlpha);
      alphas[dir] = stdMax(alphas[dir], tempAlpha);
    }
    // incrementIndices, :38-48 (x fastest)
    int dim = 0;
    for (; dim < D - 1; ++dim) {
      if (nIdx[dim] < 1) break;
      nIdx[dim] = -1;
    }
    ++nIdx[dim];
  }
  for (int i = 0; i < D; ++i)
    dissipation += alphaFactor * alpha[i] * (gradNeg[i] - gradPos[i]) * 0.5;
  return {totalGrad, dissipation};
}

// MarkVoidPoints with its default options (lsMarkVoidPoints.hpp:157-300),
// restated on grid cells: the sign field (value >= 0 or < 0, :37-39) splits
// into star-connected components over a box around the map (its bounding box
// plus 2 cells; bounded directions: the whole extent); the top component
// holds the box's last cell in HRLE order.  A defined point >= 0 is void when
// it lies outside the top component; a negative one when no neighbour of the
// other sign lies in it (:268-287).  Returns a marker per map entry.  When
// the last cell is negative nothing is marked.
template <int D> std::vector<uint8_t> voidMarkers(const LS<D> &t) {
  const Grid<D> &g = t.grid;
  std::vector<uint8_t> mark(t.keys.size(), 0);
  if (t.keys.empty()) return mark;
  int64_t lo[D], hi[D], n[D];
  for (int d = 0; d < D; ++d) lo[d] = INT64_MAX, hi[d] = INT64_MIN;
  for (uint64_t k : t.keys)
    for (int d = 0; d < D; ++d) {
      const int64_t c = coordOf<D>(k, d);
      lo[d] = std::min(lo[d], c), hi[d] = std::max(hi[d], c);
    }
  size_t N = 1;
  for (int d = 0; d < D; ++d) {
    if (g.bounded(d)) {
      lo[d] = g.minI[d];
      hi[d] = g.bc[d] == VLSG_PERIODIC_BOUNDARY ? g.maxI[d] - 1 : g.maxI[d];
    } else {
      lo[d] -= 2, hi[d] += 2;
    }
    n[d] = hi[d] - lo[d] + 1;
    N *= (size_t)n[d];
  }
  auto boxIndex = [&](const int64_t *c) {
    size_t i = 0;
    for (int d = D - 1; d >= 0; --d) i = i * n[d] + (size_t)(c[d] - lo[d]);
    return i;
  };
  std::vector<double> v(N);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)N; ++i) {
    int64_t c[D];
    size_t r = (size_t)i;
    for (int d = 0; d < D; ++d) c[d] = lo[d] + (int64_t)(r % n[d]), r /= n[d];
    v[i] = t.at(encode<D>(c));
  }
  std::vector<size_t> parent(N);
  for (size_t i = 0; i < N; ++i) parent[i] = i;
  auto find = [&](size_t x) {
    while (parent[x] != x) x = parent[x] = parent[parent[x]];
    return x;
  };
  // a neighbour inside the box (through the boundary conditions), or none
  auto neighbour = [&](const int64_t *c, int d, int s, size_t &out) {
    int64_t q[D];
    for (int e = 0; e < D; ++e) q[e] = c[e];
    q[d] = g.mapCoord(d, c[d] + s);
    if (q[d] < lo[d] || q[d] > hi[d]) return false;
    out = boxIndex(q);
    return true;
  };
  for (size_t i = 0; i < N; ++i) {
    int64_t c[D];
    size_t r = i;
    for (int d = 0; d < D; ++d) c[d] = lo[d] + (int64_t)(r % n[d]), r /= n[d];
    for (int d = 0; d < D; ++d)
      for (int s = -1; s <= 1; s += 2) {
        size_t j;
        if (!neighbour(c, d, s, j)) continue;
        if ((v[i] >= 0) != (v[j] >= 0)) continue;
        const size_t a = find(i), b = find(j);
        if (a != b) parent[std::max(a, b)] = std::min(a, b);
      }
  }
  if (v[N - 1] < 0) return mark;
  const size_t top = find(N - 1);
  for (size_t p = 0; p < t.keys.size(); ++p) {
    if (!isDefined(t.vals[p])) continue;
    int64_t c[D];
    decode<D>(t.keys[p], c);
    bool inBox = true;
    for (int d = 0; d < D; ++d) inBox = inBox && c[d] >= lo[d] && c[d] <= hi[d];
    if (!inBox) continue;
    const size_t i = boxIndex(c);
    if (t.vals[p] >= 0) {
      mark[p] = find(i) != top;
    } else {
      bool reached = false;
      for (int d = 0; d < D && !reached; ++d)
        for (int s = -1; s <= 1 && !reached; s += 2) {
          size_t j;
          if (!neighbour(c, d, s, j)) continue;
          if (std::signbit(v[j]) == std::signbit(t.vals[p])) continue;
          reached = find(j) == top;
        }
      mark[p] = !reached;
    }
  }
  return mark;
}

// Per-point rate chain of integrateTime (lsAdvect.hpp:530-588).
struct RateEntry {
  double gradient, dissipation, stop;
};

template <int D> struct Advector {
  std::vector<LS<D>> &lss; // bottom .. top
  Params P;
  VelSource vel;
  std::vector<LS<D>> initial;
  double currentTimeStep = -1.;
  uint64_t pointUpdates = 0;
  uint32_t stages = 0;

  // storedRates, in HRLE order of the active points
  std::vector<uint64_t> activeKeys;
  std::vector<int64_t> rateStart;
  std::vector<RateEntry> rates;

  Advector(std::vector<LS<D>> &l, const Params &p, const VelSource &v)
      : lss(l), P(p), vel(v) {}

  LS<D> &top() { return lss.back(); }

  // Sharding: only points with z in [ownLo, ownHi) count towards the time
  // step, the alphas and the point updates; reduceCb combines the partial
  // values over all shards (the contract of vlsg_set_owned_region and
  // vlsg_set_reduction_callback).
  bool ownZ = false;
  int64_t ownLo = 0, ownHi = 0;
  vlsg_reduce_cb reduceCb = nullptr;
  void *reduceUser = nullptr;
  bool owned(uint64_t key) const {
    if (!ownZ) return true;
    const int64_t z = coordOf<D>(key, D - 1);
    return z >= ownLo && z < ownHi;
  }
  void reduceAcross(double *v, int n, int op) {
    if (reduceCb && reduceCb(reduceUser, v, n, op) != 0)
      throw std::runtime_error("the reduction callback failed");
  }

  // findGlobalAlphas, lsAdvect.hpp:90-195
  void findGlobalAlphas(double *finalAlphas) {
    const LS<D> &t = top();
    for (int i = 0; i < D; ++i) finalAlphas[i] = 0;
    const int nt = omp_get_max_threads();
    std::vector<std::array<double, 3>> loc(nt, std::array<double, 3>{0, 0, 0});
    const std::vector<uint64_t> ids = vel.cb ? pointIds<D>(t) : std::vector<uint64_t>();
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < (int64_t)t.keys.size(); ++p) {
      const double value = t.vals[p];
      if (!isDefined(value) || std::abs(value) > Params::integrationCutoff) continue;
      const uint64_t key = t.keys[p];
      if (!owned(key)) continue;
      auto &la = loc[omp_get_thread_num()];
      for (int lower = 0; lower < (int)lss.size(); ++lower) {
        if (lss[lower].at(key) <= value + Params::wrappingLayerEpsilon) {
          double normal[3] = {0, 0, 0};
          double normalModulus = 0.;
          for (int i = 0; i < D; ++i) {
            const double phiPos = t.at(shiftKey<D>(t.grid, key, i, 1));
            const double phiNeg = t.at(shiftKey<D>(t.grid, key, i, -1));
            normal[i] = phiPos - phiNeg;
            normalModulus += normal[i] * normal[i];
          }
          normalModulus = 1. / std::sqrt(normalModulus);
          for (int i = 0; i < D; ++i) normal[i] *= normalModulus;
          double coords[3], scaVel, vecVel[3];
          coordinateOf<D>(t.grid, key, coords);
          vel.query(coords, lower, normal, vel.cb ? ids[p] : 0, scaVel, vecVel);
          for (int i = 0; i < D; ++i) {
            const double tempAlpha = std::abs((scaVel + vecVel[i]) * normal[i]);
            la[i] = stdMax(la[i], tempAlpha);
          }
          break;
        }
      }
    }
    vel.check();
    for (auto &la : loc)
      for (int i = 0; i < D; ++i) finalAlphas[i] = stdMax(finalAlphas[i], la[i]);
    reduceAcross(finalAlphas, D, VLSG_REDUCE_MAX);
  }

  // integrateTime, lsAdvect.hpp:435-612
  double integrateTime(double maxTimeStep, const double *globalAlphas) {
    LS<D> &t = top();
    activeKeys.clear();
    std::vector<int64_t> activePos;
    for (int64_t p = 0; p < (int64_t)t.keys.size(); ++p) {
      const double v = t.vals[p];
      if (isDefined(v) && std::abs(v) <= Params::integrationCutoff) {
        activeKeys.push_back(t.keys[p]);
        activePos.push_back(p);
      }
    }
    const int64_t n = activeKeys.size();
    const int L = lss.size();
    std::vector<RateEntry> chainStore(size_t(n) * L);
    std::vector<int> chainLen(n);
    const int nt = omp_get_max_threads();
    std::vector<double> tmin(nt, maxTimeStep);
    std::vector<std::array<double, 3>> alp(nt, std::array<double, 3>{0, 0, 0});
    const SchemeCtx<D> S{t, P, vel, globalAlphas};
    // setIgnoreVoids: void points get no rates (lsAdvect.hpp:443-454, :510)
    const std::vector<uint8_t> voids = P.ignoreVoids ? voidMarkers<D>(t) : std::vector<uint8_t>();
    // StencilLocalLaxFriedrichs bounds dt with the finalAlphas of its last
    // call that got past the zero-velocity return; with one thread that is
    // the last such call in HRLE order (lsAdvect.hpp:599-606)
    const bool sllf = P.spatial == VLSG_STENCIL_LOCAL_LAX_FRIEDRICHS_1ST_ORDER;
    std::vector<std::array<double, 4>> sllfLast(sllf ? n : 0, std::array<double, 4>{0, 0, 0, 0});
    const std::vector<uint64_t> ids = vel.cb ? pointIds<D>(t) : std::vector<uint64_t>();
    const double adaptiveFactor = 1.0 / P.adaptiveSubdivisions;
#pragma omp parallel for schedule(static)
    for (int64_t a = 0; a < n; ++a) {
      const int th = omp_get_thread_num();
      const uint64_t key = activeKeys[a];
      double value = t.vals[activePos[a]];
      double maxStepTime = 0;
      double cfl = P.timeStepRatio;
      int len = 0;
      RateEntry *chain = &chainStore[size_t(a) * L];
      for (int cur = L - 1; cur >= 0; --cur) {
        std::pair<double, double> gd{0., 0.};
        if (!(P.ignoreVoids && voids[activePos[a]])) {
          for (int lower = 0; lower < L; ++lower) {
            if (lss[lower].at(key) <= value + Params::wrappingLayerEpsilon) {
              double ghostAlphas[4] = {0, 0, 0, 0};
              gd = evalScheme<D>(S, key, vel.cb ? ids[activePos[a]] : 0, lower,
                                 sllf ? sllfLast[a].data()
                                      : (owned(key) ? alp[th].data() : ghostAlphas));
              break;
            }
          }
        }
        const double velocity = gd.first - gd.second;
        if (velocity > 0.) {
          maxStepTime += cfl / velocity;
          chain[len++] = {gd.first, gd.second, NEG};
          break;
        } else if (velocity == 0.) {
          maxStepTime = POS;
          chain[len++] = {gd.first, gd.second, POS};
          break;
        } else {
          double valueBelow;
          if (cur > 0)
            valueBelow = lss[cur - 1].at(key);
          else
            valueBelow = POS;
          const double difference = std::abs(valueBelow - value);
          if (difference >= cfl) {
            maxStepTime -= cfl / velocity;
            chain[len++] = {gd.first, gd.second, POS};
            break;
          } else {
            if (P.adaptiveTimeStepping && difference > adaptiveFactor * cfl) {
              maxStepTime -= adaptiveFactor * cfl / velocity;
              chain[len++] = {gd.first, gd.second, POS};
              break;
            } else {
              cfl -= difference;
              value = valueBelow;
              maxStepTime -= difference / velocity;
              chain[len++] = {gd.first, gd.second, valueBelow};
            }
          }
        }
      }
      chainLen[a] = len;
      if (owned(key) && maxStepTime < tmin[th]) tmin[th] = maxStepTime;
    }
    vel.check();
    double tempMax = maxTimeStep;
    for (int i = 0; i < nt; ++i)
      if (tmin[i] < tempMax) tempMax = tmin[i];
    if (reduceCb) {
      double m = DBL_MAX;
      for (int i = 0; i < nt; ++i)
        if (tmin[i] < m) m = tmin[i];
      reduceAcross(&m, 1, VLSG_REDUCE_MIN);
      if (m < tempMax) tempMax = m;
    }
    // reduceTimeStepHamiltonJacobi of the LF family (e.g. lsLaxFriedrichs.hpp:350-362)
    const int s = P.spatial;
    const bool lfFamily = !(s == VLSG_ENGQUIST_OSHER_1ST_ORDER ||
                            s == VLSG_ENGQUIST_OSHER_2ND_ORDER ||
                            s == VLSG_WENO_3RD_ORDER || s == VLSG_WENO_5TH_ORDER);
    if (lfFamily) {
      double fa[3] = {0, 0, 0};
      if (s == VLSG_LAX_FRIEDRICHS_1ST_ORDER || s == VLSG_LAX_FRIEDRICHS_2ND_ORDER) {
        for (int i = 0; i < D; ++i) fa[i] = globalAlphas[i];
      } else if (sllf) {
        for (int64_t a = n - 1; a >= 0; --a)
          if (sllfLast[a][3] != 0.) {
            for (int i = 0; i < D; ++i) fa[i] = sllfLast[a][i];
            break;
          }
      } else {
        for (int th = 0; th < nt; ++th)
          for (int i = 0; i < D; ++i) fa[i] = stdMax(fa[i], alp[th][i]);
        reduceAcross(fa, D, VLSG_REDUCE_MAX);
      }
      double timeStep = 0;
      for (int i = 0; i < D; ++i) timeStep += fa[i] / t.grid.delta;
      timeStep = 1.0 / timeStep;
      tempMax = stdMin(timeStep, tempMax);
    }
    if (tempMax < maxTimeStep) maxTimeStep = tempMax;
    rateStart.assign(n + 1, 0);
    for (int64_t a = 0; a < n; ++a) rateStart[a + 1] = rateStart[a] + chainLen[a];
    rates.resize(rateStart[n]);
    for (int64_t a = 0; a < n; ++a)
      for (int j = 0; j < chainLen[a]; ++j)
        rates[rateStart[a] + j] = chainStore[size_t(a) * L + j];
    return maxTimeStep;
  }

  // computeRates, lsAdvect.hpp:616-682
  bool computeRates(double maxTimeStep) {
    if (!schemeSupported(P.spatial)) return false;
    expand<D>(top(), schemeWidth(P.spatial)); // prepareLS, :973-1015
    double globalAlphas[3] = {0, 0, 0};
    if (P.spatial == VLSG_LAX_FRIEDRICHS_1ST_ORDER ||
        P.spatial == VLSG_LAX_FRIEDRICHS_2ND_ORDER)
      findGlobalAlphas(globalAlphas);
    currentTimeStep = integrateTime(maxTimeStep, globalAlphas);
    return true;
  }

  // updateLevelSet, lsAdvect.hpp:686-800
  void updateLevelSet(double dt) {
    LS<D> &t = top();
    reduce<D>(t, 1); // :700
    const bool checkDiss = P.checkDissipation;
    // after Reduce(1) the defined points are exactly the active points
    int64_t a = 0;
    for (int64_t p = 0; p < (int64_t)t.keys.size(); ++p) {
      double &value = t.vals[p];
      if (!isDefined(value)) continue;
      if (std::abs(value) > Params::integrationCutoff) continue;
      if (a >= (int64_t)activeKeys.size() || activeKeys[a] != t.keys[p])
        throw std::runtime_error("updateLevelSet: rate/point mismatch");
      const RateEntry *it = &rates[rateStart[a]];
      double time = dt;
      double velocity = it->gradient - it->dissipation;
      if ((checkDiss && (it->gradient < 0 && velocity > 0)) ||
          (it->gradient > 0 && velocity < 0))
        velocity = 0;
      double rate = time * velocity;
      while (std::abs(it->stop - value) < std::abs(rate)) {
        time -= std::abs((it->stop - value) / velocity);
        value = it->stop;
        ++it;
        velocity = it->gradient - it->dissipation;
        if ((checkDiss && (it->gradient < 0 && velocity > 0)) ||
            (it->gradient > 0 && velocity < 0))
          velocity = 0;
        rate = time * velocity;
      }
      value -= rate;
      // setSaveAdvectionVelocities: the last leg's rate and the dissipation
      // of the chain entry it ended on (lsAdvect.hpp:764-767)
      if (P.saveAdvectionVelocities && !t.pd.empty()) {
        t.pd[p].vel = rate;
        t.pd[p].diss = it->dissipation;
      }
      ++a;
    }
    if (ownZ) {
      int64_t ownedActive = 0;
      for (const uint64_t k : activeKeys) ownedActive += owned(k) ? 1 : 0;
      pointUpdates += ownedActive;
    } else {
      pointUpdates += a;
    }
    ++stages;
    t.finalizeMap();
  }

  void rebuildLS() { // :250-256
    if (P.spatial == VLSG_STENCIL_LOCAL_LAX_FRIEDRICHS_1ST_ORDER)
      rebuild<D>(top(), 1.5, 3, P.updatePointData);
    else
      rebuild<D>(top(), 1.0, 2, P.updatePointData);
  }

  void adjustLowerLayers() { // :802-813 (not with StencilLocalLaxFriedrichs)
    if (P.spatial == VLSG_STENCIL_LOCAL_LAX_FRIEDRICHS_1ST_ORDER) return;
    for (size_t i = 0; i + 1 < lss.size(); ++i)
      booleanOp<D>(lss[i], top(), maxComp);
  }

  // combineLevelSets, lsAdvect.hpp:199-236
  bool combineLevelSets(double wTarget, double wSource) {
    int steps = 1;
    if (P.temporal == VLSG_RUNGE_KUTTA_2ND_ORDER) steps = 2;
    else if (P.temporal == VLSG_RUNGE_KUTTA_3RD_ORDER) steps = 3;
    const int expansionWidth = std::ceil(2.0 * steps * P.timeStepRatio + 1);
    expand<D>(top(), expansionWidth);
    expand<D>(initial.back(), expansionWidth);
    bool movedDown = false;
    std::atomic<bool> md{false};
    booleanOp<D>(top(), initial.back(), [&](double a, double b) {
      if (a != POS && a != NEG && b != POS && b != NEG) {
        const double res = wSource * a + wTarget * b;
        if (res > b) md.store(true, std::memory_order_relaxed);
        return res;
      }
      if (a == POS || a == NEG) return a;
      return b;
    }, true, [](double a, double b) { // defined results come from A (:221-226)
      return a != POS && a != NEG && b != POS && b != NEG;
    });
    movedDown = md.load();
    rebuildLS();
    if (lss.size() > 1) {
      double m = movedDown ? 1.0 : 0.0;
      reduceAcross(&m, 1, VLSG_REDUCE_MAX);
      movedDown = m != 0.0;
    }
    return movedDown;
  }

  // AdvectTimeIntegration, lsAdvectIntegrationSchemes.hpp:46-168
  double evolveForwardEuler(double maxTimeStep, bool updateLowerLayers = true) {
    if (!computeRates(maxTimeStep)) throw std::runtime_error("scheme not supported");
    updateLevelSet(currentTimeStep);
    rebuildLS();
    if (updateLowerLayers) adjustLowerLayers();
    return currentTimeStep;
  }
  void saveInitial(bool all) {
    if (initial.size() != lss.size()) initial.resize(lss.size());
    if (all) {
      for (size_t i = 0; i < lss.size(); ++i) initial[i] = lss[i];
    } else {
      initial.back() = lss.back();
    }
  }
  void restoreLower() {
    for (size_t i = 0; i + 1 < lss.size(); ++i) lss[i] = initial[i];
  }
  // velocityUpdateCallback (lsAdvect.hpp:82, :966-969) with the top level
  // set's defined points in HRLE order (no runs)
  vlsg_update_cb updateCb = nullptr;
  void *updateUser = nullptr;
  void callUpdate() {
    LS<D> &t = top();
    std::vector<int32_t> idx;
    std::vector<double> val;
    for (size_t i = 0; i < t.keys.size(); ++i) {
      if (!isDefined(t.vals[i])) continue;
      int64_t c[D];
      decode<D>(t.keys[i], c);
      for (int d = 0; d < 3; ++d) idx.push_back(d < D ? (int32_t)c[d] : 0);
      val.push_back(t.vals[i]);
    }
    const vlsg_levelset_view v{(int64_t)val.size(), idx.data(), val.data(), 0, nullptr, nullptr,
                               t.width};
    if (updateCb(updateUser, &v) != 0) throw std::runtime_error("the velocity update callback failed");
  }
  // lsAdvectIntegrationSchemes.hpp:59-108
  double evolveRungeKutta2(double maxTimeStep) {
    const bool cb = updateCb != nullptr;
    saveInitial(cb);
    const double dt1 = evolveForwardEuler(maxTimeStep, cb);
    if (dt1 <= 0.) return 0.;
    if (cb) callUpdate();
    const double dt2 = evolveForwardEuler(dt1, false);
    const bool etched = combineLevelSets(0.5, 0.5);
    if (etched && cb) restoreLower();
    adjustLowerLayers();
    return 0.5 * dt1 + 0.5 * dt2;
  }
  // :110-168
  double evolveRungeKutta3(double maxTimeStep) {
    const bool cb = updateCb != nullptr;
    saveInitial(true);
    const double dt1 = evolveForwardEuler(maxTimeStep, cb);
    if (dt1 <= 0.) return 0.;
    if (cb) callUpdate();
    const double dt2 = evolveForwardEuler(dt1, false);
    const bool etched1 = combineLevelSets(0.75, 0.25);
    if (etched1 && cb) restoreLower();
    adjustLowerLayers();
    if (cb) callUpdate();
    const double dt3 = evolveForwardEuler(dt1, false);
    const bool etched2 = combineLevelSets(1.0 / 3.0, 2.0 / 3.0);
    if (etched2) restoreLower();
    adjustLowerLayers();
    return (dt1 + dt2 + 4.0 * dt3) / 6.0;
  }
  double advect(double maxTimeStep) { // :817-830
    switch (P.temporal) {
    case VLSG_RUNGE_KUTTA_2ND_ORDER: return evolveRungeKutta2(maxTimeStep);
    case VLSG_RUNGE_KUTTA_3RD_ORDER: return evolveRungeKutta3(maxTimeStep);
    default: return evolveForwardEuler(maxTimeStep);
    }
  }
  // apply, lsAdvect.hpp:1017-1043
  void apply(vlsg_advect_result &res) {
    // point data of the top level set: every defined point carries its own
    // index (HRLE order) into the data the caller holds
    if (P.trackPointData || P.saveAdvectionVelocities) {
      LS<D> &t = top();
      t.pd.assign(t.keys.size(), PointData{});
      int64_t r = 0;
      for (size_t i = 0; i < t.keys.size(); ++i)
        if (isDefined(t.vals[i])) t.pd[i].src = r++;
    } else {
      top().pd.clear();
    }
    double advectedTime = 0.;
    unsigned steps = 0;
    if (P.advectionTime == 0.) {
      advectedTime = advect(std::numeric_limits<double>::max());
      steps = 1;
    } else {
      double currentTime = 0.0;
      while (currentTime < P.advectionTime) {
        currentTime += advect(P.advectionTime - currentTime);
        ++steps;
        if (P.singleStep) break;
        if (steps >= P.maxSteps) throw std::runtime_error("step limit reached");
      }
      advectedTime = currentTime;
    }
    res.advected_time = advectedTime;
    res.current_time_step = currentTimeStep;
    res.number_of_time_steps = steps;
    res.number_of_stages = stages;
    res.point_updates = pointUpdates;
    res.kernel_launches = 0;
  }
};

} // namespace vlso
