// vlsg_rates.cuh -- per-active-point rates of one forward-Euler stage.
//
// Restates, per active point (defined, |phi| <= 0.5, lsAdvect.hpp:498):
//   the material choice and stop chain of integrateTime (lsAdvect.hpp:505-592),
//   the schemes' operator() -- EngquistOsher (lsEngquistOsher.hpp:42-162),
//   LaxFriedrichs (lsLaxFriedrichs.hpp:236-348), LocalLocalLaxFriedrichs
//   (lsLocalLocalLaxFriedrichs.hpp:298-421), LocalLaxFriedrichs
//   (lsLocalLaxFriedrichs.hpp:65-241), WENO3/5 (lsWENO.hpp:53-160 with
//   lsFiniteDifferences.hpp:58-123) -- and findGlobalAlphas
//   (lsAdvect.hpp:90-195), plus the per-point update of updateLevelSet
//   (lsAdvect.hpp:725-777).
// Expressions keep the reference's evaluation order; the library is compiled
// with -fmad=false so FP64 results are bit-identical to the CPU restatement.
//
// One warp per brick: the brick's active cells are found from its defined
// mask and taken 32 at a time, one thread per active point.  Stencil values
// come through the slot's 27-neighbour table, or through the brick map and
// the boundary mapping for bricks within 8 cells of a boundary that remaps
// cells.  Outputs are compact over the active points: each brick reserves
// one entry per active cell, in the order of its cell list, and the value
// update walks the same list (entry r of chain entry j at j * rateCap + r).
#pragma once

#include <type_traits>

#include "vlsg_common.cuh"
#include "vlsg_frontier.cuh"
#include "vlsg_passes.cuh"

namespace vlsg {
namespace { // internal linkage: every compilation unit has its own copy

constexpr int RATE_THREADS = 256;

template <class T> __device__ inline T sqr(T v) { return v * v; }
template <class T> __device__ inline T stdMax(T a, T b) { return (a < b) ? b : a; }
template <class T> __device__ inline T stdMin(T a, T b) { return (b < a) ? b : a; }

// vlsg_velocity_desc evaluated term by term (order fixed by vlsg.h).
template <class T>
__device__ inline T scalarVelocity(const vlsg_velocity_desc &v, int material,
                                   const T n[3]) {
  int m = material < v.n_materials ? material : v.n_materials - 1;
  if (m < 0) m = 0;
  T s = T(v.rate[m]);
  for (int k = 0; k < 3; ++k) {
    const T c = T(n[k] > 0 ? v.lin_pos[m][k] : v.lin_neg[m][k]);
    if (c != T(0)) s = s + c * n[k];
  }
  for (int k = 0; k < 3; ++k) {
    const T c = T(n[k] > 0 ? v.abs_pos[m][k] : v.abs_neg[m][k]);
    if (c != T(0)) s = s + c * fabs(n[k]);
  }
  for (int k = 0; k < 3; ++k) {
    const T c = T(n[k] > 0 ? v.sq_pos[m][k] : v.sq_neg[m][k]);
    if (c != T(0)) s = s + c * (n[k] * n[k]);
  }
  return s;
}
template <class T>
__device__ inline void vectorVelocity(const vlsg_velocity_desc &v, int material,
                                      T out[3]) {
  int m = material < v.n_materials ? material : v.n_materials - 1;
  if (m < 0) m = 0;
  for (int k = 0; k < 3; ++k) out[k] = T(v.vec[m][k]);
}

// Velocity of one evaluation site of an active point (site 0: the point
// itself; LocalLaxFriedrichs site 1 + q: box neighbour q, x fastest).
// FunctorVel evaluates the device functor; TableVel reads what the host
// callback returned for this point (entry material * sites + site).
// alpha(dir, material, cd, q): getDissipationAlpha at box neighbour q
// (LocalLaxFriedrichsAnalytical).
struct FunctorVel {
  const vlsg_velocity_desc &d;
  template <class T>
  __device__ void get(int material, const T n[3], int site, T &sv, T vv[3]) const {
    (void)site;
    sv = scalarVelocity<T>(d, material, n);
    vectorVelocity<T>(d, material, vv);
  }
  template <class T> __device__ T alpha(int dir, int material, const T cd[3], int q) const {
    (void)cd, (void)q;
    int m = material < d.n_materials ? material : d.n_materials - 1;
    if (m < 0) m = 0;
    return T(d.alpha[m][dir]);
  }
};
struct TableVel {
  const double *s, *v;
  size_t base;
  int sites;
  const double *a; // alphas: ((p * L + material) * 27 + q) * 3 + dir, or none
  size_t alphaBase;
  // StencilLocalLaxFriedrichs: sites 28.. (nudged normals, scalar only) at
  // (p * L + material) * 162 + site - 28
  const double *s2;
  size_t base2;
  template <class T>
  __device__ void get(int material, const T n[3], int site, T &sv, T vv[3]) const {
    (void)n;
    if (site >= 28) {
      sv = T(s2[base2 + (size_t)material * 162 + (site - 28)]);
      vv[0] = vv[1] = vv[2] = T(0);
      return;
    }
    const size_t i = base + (size_t)material * sites + site;
    sv = T(s[i]);
    for (int k = 0; k < 3; ++k) vv[k] = T(v[3 * i + k]);
  }
  template <class T> __device__ T alpha(int dir, int material, const T cd[3], int q) const {
    (void)cd;
    return a ? T(a[alphaBase + ((size_t)material * 27 + q) * 3 + dir]) : T(0);
  }
};

template <class T> struct RateArgs {
  GridDev g;
  MapView m;
  Buf<T> ls[VLSG_MAX_LEVEL_SETS];
  int L;
  const int *slotList, *nSlots;
  const int *nbr;       // 27-neighbour table per slot
  const uint8_t *cflag; // CF_* per slot
  const uint64_t *def;  // defined masks of the top level set
  uint64_t *act;        // out: active masks of the top level set
  int scheme;
  double cfl;
  double dissipationAlpha;
  int calcNormals;
  int adaptive;
  double adaptiveFactor;
  int checkDiss;
  T globalAlpha[3];
  // outputs, compact over the active points: a brick reserves one entry per
  // active cell (rateNext) and records where they start (rateBase[slot]);
  // chain entry j of entry r is at j * rateCap + r, in the order of the
  // brick's active cells
  T *rateV;
  T *rateStop;
  T *rateD; // the dissipation per chain entry (setSaveAdvectionVelocities), or null
  uint8_t *rateLen;
  size_t rateCap;
  unsigned long long *rateNext;
  unsigned long long *rateBase;
  int rateOverflowErr; // err bit for a brick left out (0: the host checks rateNext)
  unsigned long long *minStep;  // bits of the smallest non-negative step
  unsigned long long *alphaMax; // bits of the LLF/LLLF alphas
  unsigned long long *counts;   // out: active cells, band cells
  int *err;
  // host callback mode: active points before list entry w, and the
  // velocities of point p at (p * L + material) * velSites + site
  const uint32_t *actOff;
  const double *velS, *velV;
  int velSites;
  const double *alphaTab; // LocalLaxFriedrichsAnalytical: the alpha callback's answers
  const double *velS2;    // StencilLocalLaxFriedrichs: the nudged-normal answers
  // StencilLocalLaxFriedrichs: baseNormalEpsilon, the dissipation limit, and
  // per warp the last (HRLE order) call's finalAlphas: key, alphas
  double sllfEps;
  double maxDissipation;
  unsigned long long *sllfKey;
  double *sllfAlpha;
  // setIgnoreVoids: void bits of the top level set (no rates there), or none
  const uint64_t *voidMask;
  // sharding: only points with z in [ownLo, ownHi) count towards the time
  // step, the alphas and the point updates (ownZ false: every point)
  bool ownZ;
  int ownLo, ownHi;
  // batching form (slotDom non-null): per slot its domain; per domain its
  // gridDelta and velocity functor, and this pass's reductions (RED_* words
  // per domain: smallest step bits, alpha bits x3, active cells) in place of
  // minStep / alphaMax / counts
  const int *slotDom;
  const double *domDelta;
  const vlsg_velocity_desc *domVel;
  unsigned long long *domRed;
};
constexpr int RED_MIN = 0, RED_ALPHA = 1, RED_ACTIVE = 4, RED_WORDS = 5;

// Reader of the top level set around one active point.
template <class T> struct Stencil {
  const GridDev &g;
  const MapView &m;
  const Buf<T> &b;
  int slot, lx, ly, lz, x0, y0, z0;
  __device__ T at(int dx, int dy, int dz) const {
    const int nx = lx + dx, ny = ly + dy, nz = lz + dz;
    if ((unsigned)nx < 8u && (unsigned)ny < 8u && (unsigned)nz < 8u &&
        cellExists(g, x0 + nx, y0 + ny, z0 + nz))
      return b.vals[(size_t)slot * BV + (nz * 64 + ny * 8 + nx)];
    return cellValueRaw<T>(g, m, b, x0 + nx, y0 + ny, z0 + nz);
  }
  __device__ T axis(int d, int off) const {
    return d == 0 ? at(off, 0, 0) : (d == 1 ? at(0, off, 0) : at(0, 0, off));
  }
};

// Reader of the top level set around one active point through the slot's
// 27-neighbour table (offsets up to 8 cells; every cell it reaches exists and
// is not remapped by a boundary).
template <class T> struct TableStencil {
  const T *vals;
  const int8_t *farSign;
  const int *nb27;
  int lx, ly, lz;
  __device__ T at(int dx, int dy, int dz) const {
    const int nx = lx + dx, ny = ly + dy, nz = lz + dz;
    const int ref = nb27[((nz >> 3) + 1) * 9 + ((ny >> 3) + 1) * 3 + ((nx >> 3) + 1)];
    if (ref < 0) return farSign[-1 - ref] < 0 ? Lim<T>::lowest() : Lim<T>::max();
    return vals[(size_t)ref * BV + ((nz & 7) * 64 + (ny & 7) * 8 + (nx & 7))];
  }
  __device__ T axis(int d, int off) const {
    return d == 0 ? at(off, 0, 0) : (d == 1 ? at(0, off, 0) : at(0, 0, off));
  }
};

template <class T, class St>
__device__ inline void oneSided(const St &S, int i, T phi0, T gridDelta,
                                int order, T &diffPos, T &diffNeg) {
  const T deltaPos = gridDelta;
  const T deltaNeg = -gridDelta;
  const T phiPos = S.axis(i, 1);
  const T phiNeg = S.axis(i, -1);
  diffPos = (phiPos - phi0) / deltaPos;
  diffNeg = (phiNeg - phi0) / deltaNeg;
  if (order == 2) {
    const T deltaPosPos = 2 * gridDelta;
    const T deltaNegNeg = -2 * gridDelta;
    const T phiPosPos = S.axis(i, 2);
    const T phiNegNeg = S.axis(i, -2);
    const T diff00 =
        (((deltaNeg * phiPos - deltaPos * phiNeg) / (deltaPos - deltaNeg) + phi0)) /
        (deltaPos * deltaNeg);
    const T diffNegNeg = (((deltaNeg * phiNegNeg - deltaNegNeg * phiNeg) /
                               (deltaNegNeg - deltaNeg) +
                           phi0)) /
                         (deltaNegNeg * deltaNeg);
    const T diffPosPos = (((deltaPos * phiPosPos - deltaPosPos * phiPos) /
                               (deltaPosPos - deltaPos) +
                           phi0)) /
                         (deltaPosPos * deltaPos);
    if (signbit(diff00) == signbit(diffPosPos)) {
      if (fabs(diffPosPos * deltaPos) < fabs(diff00 * deltaNeg))
        diffPos -= deltaPos * diffPosPos;
      else
        diffPos += deltaNeg * diff00;
    }
    if (signbit(diff00) == signbit(diffNegNeg)) {
      if (fabs(diffNegNeg * deltaNeg) < fabs(diff00 * deltaPos))
        diffNeg -= deltaNeg * diffNegNeg;
      else
        diffNeg += deltaPos * diff00;
    }
  }
}

template <class T>
__device__ inline T weno3(const T *x, T delta, bool plus) {
  const T eps = T(1e-6);
  T d0, d1, d2;
  if (plus) {
    d0 = x[2] - x[1];
    d1 = x[3] - x[2];
    d2 = x[4] - x[3];
    const T N = eps + sqr(d2 - d1);
    const T Dd = eps + sqr(d1 - d0);
    const T D2 = Dd * Dd;
    const T wp = D2 / (D2 + 2 * N * N);
    return (d0 + d1 - wp * (d2 - 2 * d1 + d0)) / (2 * delta);
  }
  d0 = x[1] - x[0];
  d1 = x[2] - x[1];
  d2 = x[3] - x[2];
  const T N = eps + sqr(d1 - d0);
  const T Dd = eps + sqr(d2 - d1);
  const T D2 = Dd * Dd;
  const T wp = D2 / (D2 + 2 * N * N);
  return (d1 + d2 - wp * (d0 - 2 * d1 + d2)) / (2 * delta);
}

template <class T>
__device__ inline T weno5(const T *x, T dx, bool plus) {
  const T eps = T(1e-6);
  T d[5];
  if (!plus) {
#pragma unroll
    for (int i = 0; i < 5; ++i) d[i] = x[i + 1] - x[i];
  } else {
#pragma unroll
    for (int i = 0; i < 5; ++i) d[i] = x[6 - i] - x[5 - i];
  }
  const T c1312 = T(13.0 / 12.0), c14 = T(1.0 / 4.0), c16 = T(1.0 / 6.0);
  const T s1 = c1312 * sqr(d[0] - 2 * d[1] + d[2]) + c14 * sqr(d[0] - 4 * d[1] + 3 * d[2]);
  const T s2 = c1312 * sqr(d[1] - 2 * d[2] + d[3]) + c14 * sqr(d[1] - d[3]);
  const T s3 = c1312 * sqr(d[2] - 2 * d[3] + d[4]) + c14 * sqr(3 * d[2] - 4 * d[3] + d[4]);
  const T eps_scaled = eps * dx * dx;
  const T al1 = T(0.1) / (eps_scaled + s1);
  const T al2 = T(0.6) / (eps_scaled + s2);
  const T al3 = T(0.3) / (eps_scaled + s3);
  const T alsum = al1 + al2 + al3;
  const T p1 = c16 * (2 * d[0] - 7 * d[1] + 11 * d[2]);
  const T p2 = c16 * (-d[1] + 5 * d[2] + 2 * d[3]);
  const T p3 = c16 * (2 * d[2] + 5 * d[3] - d[4]);
  return (al1 * p1 + al2 * p2 + al3 * p3) / (alsum * dx);
}

// Central differences at box neighbour q (x fastest):
// calculateNormalComponent of lsLocalLaxFriedrichsAnalytical.hpp:30-34.
template <class T, class St>
__device__ inline void boxDifferences(const St &S, T gridDelta, int q, T cd[3]) {
  const int ox = q % 3 - 1, oy = (q / 3) % 3 - 1, oz = q / 9 - 1;
  const T center = S.at(ox, oy, oz);
  for (int dir = 0; dir < 3; ++dir) {
    const T neg = S.at(ox - (dir == 0), oy - (dir == 1), oz - (dir == 2));
    const T pos = S.at(ox + (dir == 0), oy + (dir == 1), oz + (dir == 2));
    const T diffPos = (pos - center) / gridDelta;
    const T diffNeg = (center - neg) / gridDelta;
    cd[dir] = (diffPos + diffNeg) * T(0.5);
  }
}

// StencilLocalLaxFriedrichsScalar's FIRST_ORDER gradient component i at
// box offset (ox, oy, oz): the three values along i are taken with
// coordinate i set to -1, 0, 1 whatever the offset's (calculateGradient /
// calculateNormal, lsStencilLocalLaxFriedrichsScalar.hpp:336-378;
// FiniteDifferences, lsFiniteDifferences.hpp:132-181).
template <class T, class St>
__device__ inline T sllfGrad(const St &S, double delta, int ox, int oy, int oz, int i) {
  T v[3];
  for (int j = 0; j < 3; ++j)
    v[j] = S.at(i == 0 ? j - 1 : ox, i == 1 ? j - 1 : oy, i == 2 ? j - 1 : oz);
  const T dNeg = T((v[1] - v[0]) / delta);
  const T dPos = T((v[2] - v[1]) / delta);
  return T((dPos + dNeg) * 0.5);
}
template <class T, class St>
__device__ inline void sllfNormal(const St &S, double delta, int ox, int oy, int oz, T n[3]) {
  T modulus = 0.;
  for (int i = 0; i < 3; ++i) {
    n[i] = sllfGrad<T>(S, delta, ox, oy, oz, i);
    modulus += n[i] * n[i];
  }
  modulus = T(1) / sqrt(modulus);
  for (int i = 0; i < 3; ++i) n[i] *= modulus;
}
// calculateSimpleAdaptiveEpsilon (ADAPTIVE_EPSILON_STRATEGY 1, :60-75)
template <class T> __device__ inline T sllfEpsilon(T velocity, double baseNormalEpsilon, double delta) {
  const T absVel = fabs(velocity);
  const T baseEps = T(baseNormalEpsilon * delta);
  if (absVel > T(1e-10)) {
    const T scale = stdMax(T(0.1), stdMin(T(10.0), absVel));
    return baseEps * scale;
  }
  return baseEps;
}

// StencilLocalLaxFriedrichsScalar<T,3,1>::operator() (:219-400).  Velocity
// sites: 0 the point, 1 + q the stencil point q (x fastest), 28 + 6q + 2k
// (+1) the normal of q nudged by -DN (+DN) along k.  alphas[0..2] receive
// this call's finalAlphas and alphas[3] = 1 when the call gets past the
// zero-velocity return.
template <class T, class St, class Vel>
__device__ void evalStencilLLF(const RateArgs<T> &A, const Vel &vel, const St &S, int material,
                               T *alphas, T &outG, T &outD) {
  const double delta = A.g.delta;
  T normalVector[3];
  sllfNormal<T>(S, delta, 0, 0, 0, normalVector);
  T sv0, vv0[3];
  vel.get(material, normalVector, 0, sv0, vv0);
  double scalarVelocity = (double)sv0;
  for (int i = 0; i < 3; ++i) scalarVelocity += (double)(vv0[i] * normalVector[i]);
  if (scalarVelocity == 0.) {
    outG = 0;
    outD = 0;
    return;
  }
  T gradSq = 0;
  for (int i = 0; i < 3; ++i) {
    const T gi = sllfGrad<T>(S, delta, 0, 0, 0, i);
    gradSq += gi * gi;
  }
  const T hamiltonian = T((double)sqrt(gradSq) * scalarVelocity);
  T maxAlpha[3] = {0, 0, 0};
  // D = 2 (the plane of a z-periodic grid): the 3x3 stencil of the plane and
  // the normal nudged in x and y only, as the 2D reference does; the z terms
  // below then add exact zeros
  const bool planar = A.g.planar != 0;
  const int nSt = planar ? 9 : 27, nDir = planar ? 2 : 3;
  int cx = -1, cy = -1, cz = planar ? 0 : -1;
  for (int st = 0; st < nSt; ++st) {
    T ln[3];
    sllfNormal<T>(S, delta, cx, cy, cz, ln);
    // a corrupted normal leaves the stencil index where it is (:288-293)
    if (fabs(ln[0]) < T(1e-6) && fabs(ln[1]) < T(1e-6) && fabs(ln[2]) < T(1e-6)) continue;
    const int q = (cz + 1) * 9 + (cy + 1) * 3 + (cx + 1);
    T lsv, lvv[3];
    vel.get(material, ln, 1 + q, lsv, lvv);
    for (int dir = 0; dir < 3; ++dir) lsv += lvv[dir] * ln[dir];
    const T DN = sllfEpsilon<T>(lsv, A.sllfEps, delta);
    T np[3] = {ln[0], ln[1], ln[2]}, nn[3] = {ln[0], ln[1], ln[2]}, vd[3] = {0, 0, 0};
    for (int k = 0; k < nDir; ++k) {
      np[k] -= DN;
      nn[k] += DN;
      T vp, vn, unused[3];
      vel.get(material, np, 28 + 6 * q + 2 * k, vp, unused);
      vel.get(material, nn, 28 + 6 * q + 2 * k + 1, vn, unused);
      vd[k] = T((double)(vn - vp) / (2.0 * (double)DN));
      np[k] += DN;
      nn[k] -= DN;
    }
    T gr[3];
    for (int i = 0; i < 3; ++i) gr[i] = sllfGrad<T>(S, delta, cx, cy, cz, i);
    T denom = 0;
    for (int i = 0; i < 3; ++i) denom += gr[i] * gr[i];
    for (int k = 0; k < 3; ++k) {
      T monti = 0, toifl = 0;
      for (int j = 0; j < 2; ++j) {
        const int idx = (k + 1 + j) % 3;
        monti += gr[idx] * gr[idx];
        toifl += gr[idx] * vd[idx];
      }
      monti *= vd[k] / denom;
      toifl *= -gr[k] / denom;
      const T osher = lsv * ln[k];
      maxAlpha[k] = stdMax(maxAlpha[k], T(fabs(monti + toifl + osher)));
    }
    // incrementIndex, x fastest (:196-204)
    if (cx < 1) {
      ++cx;
    } else {
      cx = -1;
      if (cy < 1) {
        ++cy;
      } else {
        cy = -1;
        ++cz;
      }
    }
  }
  T dissipation = 0.;
  for (int d = 0; d < 3; ++d) {
    T v[3];
    for (int j = 0; j < 3; ++j) v[j] = S.at(d == 0 ? j - 1 : 0, d == 1 ? j - 1 : 0, d == 2 ? j - 1 : 0);
    const T dNeg = T((v[1] - v[0]) / delta);
    const T dPos = T((v[2] - v[1]) / delta);
    const T gradientDiff = T((dPos - dNeg) * 0.5);
    const T finalAlpha = stdMin(maxAlpha[d], T(A.maxDissipation));
    alphas[d] = finalAlpha;
    dissipation += finalAlpha * gradientDiff;
  }
  alphas[3] = T(1);
  outG = hamiltonian;
  outD = dissipation;
}

// One scheme evaluation (Hamiltonian, dissipation) for `material`.
// Scheme families a rate kernel is compiled for: every scheme but the
// stencil one (chosen at run time), WENO only, StencilLocalLaxFriedrichs only.
enum : int { FAM_ANY = 0, FAM_WENO = 1, FAM_STENCIL = 2 };

template <class T, class St, class Vel, int FAM = FAM_ANY>
__device__ void evalScheme(const RateArgs<T> &A, const Vel &vel,
                           const St &S, T C, int material, T *alphas,
                           T &outG, T &outD, double delta) {
  if constexpr (FAM == FAM_STENCIL) {
    (void)C;
    evalStencilLLF<T>(A, vel, S, material, alphas, outG, outD);
    return;
  }
  const T gridDelta = T(delta);
  const int sch = A.scheme;
  if (FAM == FAM_WENO || sch == VLSG_WENO_3RD_ORDER || sch == VLSG_WENO_5TH_ORDER) {
    const int r = sch == VLSG_WENO_3RD_ORDER ? 2 : 3;
    T gradPosTotal = 0, gradNegTotal = 0;
    T wMinus[3], wPlus[3], st[7];
    for (int i = 0; i < 3; i++) {
      st[r] = C;
      for (int k = 1; k <= r; ++k) {
        st[r + k] = S.axis(i, k);
        st[r - k] = S.axis(i, -k);
      }
      if (r == 2) {
        wMinus[i] = weno3<T>(st, gridDelta, false);
        wPlus[i] = weno3<T>(st, gridDelta, true);
      } else {
        wMinus[i] = weno5<T>(st, gridDelta, false);
        wPlus[i] = weno5<T>(st, gridDelta, true);
      }
      gradPosTotal += sqr(stdMax(wMinus[i], T(0))) + sqr(stdMin(wPlus[i], T(0)));
      gradNegTotal += sqr(stdMin(wMinus[i], T(0))) + sqr(stdMax(wPlus[i], T(0)));
    }
    T vel_grad = 0.;
    T n[3] = {0, 0, 0};
    // the scheme receives dissipationAlpha as its calcNormal flag
    if (A.dissipationAlpha != 0.0) {
      T denominator = 0;
      for (int i = 0; i < 3; i++) {
        const T pos = S.axis(i, 1);
        const T neg = S.axis(i, -1);
        n[i] = pos - neg;
        denominator += n[i] * n[i];
      }
      if (denominator > 0) {
        denominator = T(1.) / sqrt(denominator);
        for (int i = 0; i < 3; ++i) n[i] *= denominator;
      }
    }
    T sv, vv[3];
    vel.get(material, n, 0, sv, vv);
    if (sv > 0)
      vel_grad += sqrt(gradPosTotal) * sv;
    else
      vel_grad += sqrt(gradNegTotal) * sv;
    for (int w = 0; w < 3; w++) {
      if (vv[w] > T(0))
        vel_grad += vv[w] * wMinus[w];
      else
        vel_grad += vv[w] * wPlus[w];
    }
    outG = vel_grad;
    outD = 0;
    return;
  }
  if constexpr (FAM == FAM_WENO) {
    return;
  } else {
  const int order = (sch == VLSG_ENGQUIST_OSHER_2ND_ORDER ||
                     sch == VLSG_LAX_FRIEDRICHS_2ND_ORDER ||
                     sch == VLSG_LOCAL_LOCAL_LAX_FRIEDRICHS_2ND_ORDER ||
                     sch == VLSG_LOCAL_LAX_FRIEDRICHS_2ND_ORDER)
                        ? 2
                        : 1;
  T gradPos[3], gradNeg[3];
  if (sch == VLSG_ENGQUIST_OSHER_1ST_ORDER || sch == VLSG_ENGQUIST_OSHER_2ND_ORDER) {
    T gradPosTotal = 0, gradNegTotal = 0;
    for (int i = 0; i < 3; i++) {
      T diffPos, diffNeg;
      oneSided<T>(S, i, C, gridDelta, order, diffPos, diffNeg);
      gradPos[i] = diffNeg;
      gradNeg[i] = diffPos;
      gradPosTotal += sqr(stdMax(diffNeg, T(0))) + sqr(stdMin(diffPos, T(0)));
      gradNegTotal += sqr(stdMin(diffNeg, T(0))) + sqr(stdMax(diffPos, T(0)));
    }
    T vel_grad = 0.;
    T n[3] = {0, 0, 0};
    if (A.calcNormals) {
      T denominator = 0;
      for (int i = 0; i < 3; i++) {
        const T pos = S.axis(i, 1) - C;
        const T neg = C - S.axis(i, -1);
        n[i] = (pos + neg) * T(0.5);
        denominator += n[i] * n[i];
      }
      denominator = T(1.) / sqrt(denominator);
      for (int i = 0; i < 3; ++i) n[i] *= denominator;
    }
    T sv, vv[3];
    vel.get(material, n, 0, sv, vv);
    if (sv > 0)
      vel_grad += sqrt(gradPosTotal) * sv;
    else
      vel_grad += sqrt(gradNegTotal) * sv;
    for (int w = 0; w < 3; w++) {
      if (vv[w] > T(0))
        vel_grad += vv[w] * gradPos[w];
      else
        vel_grad += vv[w] * gradNeg[w];
    }
    outG = vel_grad;
    outD = 0;
    return;
  }
  const bool globalLF = (sch == VLSG_LAX_FRIEDRICHS_1ST_ORDER ||
                         sch == VLSG_LAX_FRIEDRICHS_2ND_ORDER);
  const bool calcNormal = globalLF ? (A.calcNormals != 0) : true;
  const T alphaFactor = T(A.dissipationAlpha);
  T grad = 0., dissipation = 0.;
  T n[3] = {0, 0, 0};
  T normalModulus = 0;
  for (int i = 0; i < 3; i++) {
    T diffPos, diffNeg;
    oneSided<T>(S, i, C, gridDelta, order, diffPos, diffNeg);
    gradPos[i] = diffNeg;
    gradNeg[i] = diffPos;
    if (calcNormal) {
      n[i] = (diffNeg + diffPos) * T(0.5);
      normalModulus += n[i] * n[i];
    }
    grad += sqr((diffNeg + diffPos) * T(0.5));
    if (globalLF)
      dissipation += alphaFactor * A.globalAlpha[i] * (diffPos - diffNeg) * T(0.5);
  }
  if (calcNormal) {
    normalModulus = T(1.) / sqrt(normalModulus);
    for (int i = 0; i < 3; ++i) n[i] *= normalModulus;
  }
  T sv, vv[3];
  vel.get(material, n, 0, sv, vv);
  T totalGrad = 0.;
  if (sv != T(0)) totalGrad = sv * sqrt(grad);
  for (int w = 0; w < 3; w++) {
    if (vv[w] > T(0))
      totalGrad += vv[w] * gradPos[w];
    else
      totalGrad += vv[w] * gradNeg[w];
  }
  if (globalLF) {
    outG = totalGrad;
    outD = (totalGrad != T(0)) ? dissipation : T(0);
    return;
  }
  if (totalGrad == T(0)) {
    outG = 0;
    outD = 0;
    return;
  }
  if (sch == VLSG_LOCAL_LAX_FRIEDRICHS_ANALYTICAL_1ST_ORDER) {
    // the user's alphas over the 3x3x3 box at the central differences
    // (calculateNormalComponent, not normalised), no alphaFactor
    // (D = 2, the plane of a z-periodic grid: the plane's 3x3 box and the
    // directions x and y, as the 2D reference asks them)
    T alpha[3] = {0, 0, 0};
    const int q0 = A.g.planar ? 9 : 0, q1 = A.g.planar ? 18 : 27, nDir = A.g.planar ? 2 : 3;
    for (int q = q0; q < q1; ++q) {
      T cd[3];
      boxDifferences<T>(S, gridDelta, q, cd);
      for (int dir = 0; dir < nDir; ++dir) {
        const T tempAlpha = vel.alpha(dir, material, cd, q);
        alpha[dir] = stdMax(alpha[dir], tempAlpha);
        alphas[dir] = stdMax(alphas[dir], tempAlpha);
      }
    }
    for (int i = 0; i < 3; ++i) dissipation += alpha[i] * (gradNeg[i] - gradPos[i]) * T(0.5);
    outG = totalGrad;
    outD = dissipation;
    return;
  }
  if (sch == VLSG_LOCAL_LOCAL_LAX_FRIEDRICHS_1ST_ORDER ||
      sch == VLSG_LOCAL_LOCAL_LAX_FRIEDRICHS_2ND_ORDER) {
    for (int i = 0; i < 3; ++i) {
      const T alpha = fabs((sv + vv[i]) * n[i]);
      alphas[i] = stdMax(alphas[i], alpha);
      dissipation += alphaFactor * alpha * (gradNeg[i] - gradPos[i]) * T(0.5);
    }
    outG = totalGrad;
    outD = dissipation;
    return;
  }
  // LocalLaxFriedrichs: alphas over the 3x3x3 box, x fastest (D = 2: the
  // plane's 3x3 box, q 9..17)
  T alpha[3] = {0, 0, 0};
  const int q1 = A.g.planar ? 18 : 27;
  for (int q = A.g.planar ? 9 : 0; q < q1; ++q) {
    const int ox = q % 3 - 1, oy = (q / 3) % 3 - 1, oz = q / 9 - 1;
    T normal[3];
    T nm = 0.;
    const T center = S.at(ox, oy, oz);
    for (int dir = 0; dir < 3; ++dir) {
      const T neg = S.at(ox - (dir == 0), oy - (dir == 1), oz - (dir == 2));
      const T pos = S.at(ox + (dir == 0), oy + (dir == 1), oz + (dir == 2));
      const T dPos = (pos - center) / gridDelta;
      const T dNeg = (center - neg) / gridDelta;
      normal[dir] = (dPos + dNeg) * T(0.5);
      nm += normal[dir] * normal[dir];
    }
    nm = T(1.) / sqrt(nm);
    for (int dir = 0; dir < 3; ++dir) normal[dir] *= nm;
    T scaVel, vecVel[3];
    vel.get(material, normal, 1 + q, scaVel, vecVel);
    for (int dir = 0; dir < 3; ++dir) {
      const T tempAlpha = fabs((scaVel + vecVel[dir]) * normal[dir]);
      alpha[dir] = stdMax(alpha[dir], tempAlpha);
      alphas[dir] = stdMax(alphas[dir], tempAlpha);
    }
  }
  for (int i = 0; i < 3; ++i)
    dissipation += alphaFactor * alpha[i] * (gradNeg[i] - gradPos[i]) * T(0.5);
  outG = totalGrad;
  outD = dissipation;
  }
}

template <class T>
__device__ inline T lsValueAt(const Buf<T> &b, int slot, int c) {
  return b.vals[(size_t)slot * BV + c];
}

// Bits of a per-point step for the minimum (v >= 0; NaN or "no point" -1
// never lowers the minimum, lsAdvect.hpp:591) and of an alpha for the maximum.
__device__ inline unsigned long long stepBits(double v) {
  return (v >= 0.0) ? orderedBits(v + 0.0) : ~0ull;
}
__device__ inline unsigned long long alphaBits(double v) {
  return (v > 0.0) ? orderedBits(v) : 0ull;
}
__device__ inline unsigned long long warpMinU64(unsigned long long b) {
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long t = __shfl_xor_sync(0xffffffffu, b, o);
    b = t < b ? t : b;
  }
  return b;
}
__device__ inline unsigned long long warpMaxU64(unsigned long long b) {
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long t = __shfl_xor_sync(0xffffffffu, b, o);
    b = t > b ? t : b;
  }
  return b;
}

// integrateTime for one active point (lsAdvect.hpp:501-592): the material
// chain, the stored rates (velocity as updateLevelSet applies it,
// lsAdvect.hpp:738-744, and the stop value) and the point's time budget.
template <class T, class St, class Vel, int FAM = FAM_ANY>
__device__ inline double ratePoint(const RateArgs<T> &A, const Vel &vel,
                                   const St &S, int slot, int c, T C, T *alphas,
                                   double delta, size_t q) {
  const int L = A.L;
  T value = C;
  double maxStepTime = 0;
  double cfl = A.cfl;
  int len = 0;
  const bool isVoid = A.voidMask && ((A.voidMask[(size_t)slot * 8 + (c >> 6)] >> (c & 63)) & 1ull);
  for (int cur = L - 1; cur >= 0; --cur) {
    T g = 0, d = 0;
    for (int lower = 0; lower < L && !isVoid; ++lower) {
      const T lv = lower == L - 1 ? C : lsValueAt<T>(A.ls[lower], slot, c);
      if ((double)lv <= (double)value + 1e-4) {
        evalScheme<T, St, Vel, FAM>(A, vel, S, C, lower, alphas, g, d, delta);
        break;
      }
    }
    const T velocity = g - d;
    T veff = velocity;
    if ((A.checkDiss && (g < 0 && velocity > 0)) || (g > 0 && velocity < 0)) veff = 0;
    T stop;
    bool done = true;
    if (velocity > 0.) {
      maxStepTime += cfl / velocity;
      stop = Lim<T>::lowest();
    } else if (velocity == 0.) {
      maxStepTime = (double)Lim<T>::max();
      stop = Lim<T>::max();
    } else {
      const T valueBelow = cur > 0 ? lsValueAt<T>(A.ls[cur - 1], slot, c) : Lim<T>::max();
      const T difference = fabs(valueBelow - value);
      if ((double)difference >= cfl) {
        maxStepTime -= cfl / velocity;
        stop = Lim<T>::max();
      } else if (A.adaptive && (double)difference > A.adaptiveFactor * cfl) {
        maxStepTime -= A.adaptiveFactor * cfl / velocity;
        stop = Lim<T>::max();
      } else {
        cfl -= difference;
        value = valueBelow;
        maxStepTime -= difference / velocity;
        stop = valueBelow;
        done = false;
      }
    }
    A.rateV[(size_t)len * A.rateCap + q] = veff;
    A.rateStop[(size_t)len * A.rateCap + q] = stop;
    if (A.rateD) A.rateD[(size_t)len * A.rateCap + q] = d;
    ++len;
    if (done) break;
  }
  A.rateLen[q] = (uint8_t)len;
  return maxStepTime;
}

// Stencil of local cell c of `slot`: the table reader, or the global one
// near a boundary that remaps cells; fn(stencil, centre value).
template <class T, class Fn>
__device__ inline void withStencil(const RateArgs<T> &A, int slot, int c, Fn fn) {
  const Buf<T> &top = A.ls[A.L - 1];
  const T C = top.vals[(size_t)slot * BV + c];
  if (A.cflag[slot] & CF_NEAR) {
    int bx, by, bz;
    brickCoords(A.g, A.m.slotBrick[slot], bx, by, bz);
    const Stencil<T> S{A.g, A.m, top, slot, c & 7, (c >> 3) & 7, c >> 6,
                       A.g.org[0] + bx * BS, A.g.org[1] + by * BS, A.g.org[2] + bz * BS};
    fn(S, C);
  } else {
    const TableStencil<T> S{top.vals, top.farSign, A.nbr + (size_t)slot * 27, c & 7,
                            (c >> 3) & 7, c >> 6};
    fn(S, C);
  }
}

// Active mask of a brick (defined cells with |phi| <= 0.5, lsAdvect.hpp:498;
// lane z returns plane z): one coalesced read of the brick's 512 values.
template <class T>
__device__ inline uint64_t activePlanes(const T *vals, int slot) {
  const int lane = threadIdx.x & 31;
  const T *p = vals + (size_t)slot * BV + lane;
  T v[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = p[32 * i];
  uint64_t mine = 0;
#pragma unroll
  for (int z = 0; z < 8; ++z) {
    const unsigned lo = __ballot_sync(0xffffffffu, isDef(v[2 * z]) && fabs(v[2 * z]) <= T(0.5));
    const unsigned hi =
        __ballot_sync(0xffffffffu, isDef(v[2 * z + 1]) && fabs(v[2 * z + 1]) <= T(0.5));
    if (lane == z) mine = (uint64_t)lo | ((uint64_t)hi << 32);
  }
  return mine;
}

// Resident blocks per SM: 3 for float (80 registers), 4 for the float WENO
// kernels (64 registers: a few spilled values, 8% faster than 3 blocks), 2
// for double (the FP64 stencils need 128 registers to stay out of local
// memory).
template <class T, int FAM = FAM_ANY> constexpr int rateMinBlocks() {
  return sizeof(T) == 4 ? (FAM == FAM_WENO ? 4 : 3) : 2;
}
// MODE 0: rates (integrateTime); MODE 1: the global alphas of the
// Lax-Friedrichs schemes (findGlobalAlphas).  TABLE: velocities from the
// host callback's table instead of the device functor.
// BATCH: the batching form (per-domain spacing, velocity and reductions,
// A.slotDom set).
// MINB: resident blocks per SM to compile for (0: rateMinBlocks), the launch
// shapes the batching form's autotuner chooses from.
template <class T, int MODE, bool TABLE = false, int FAM = FAM_ANY, bool BATCH = false, int MINB = 0>
__global__ void __launch_bounds__(RATE_THREADS, MINB ? MINB : rateMinBlocks<T, FAM>())
    kRates(RateArgs<T> A, const vlsg_velocity_desc desc) {
  __shared__ uint16_t sList[RATE_THREADS / 32][BV];
  uint16_t *list = sList[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nWarps = (gridDim.x * blockDim.x) >> 5;
  const int n = *A.nSlots;
  const int L = A.L;
  const Buf<T> &top = A.ls[L - 1];
  unsigned long long minBits = ~0ull, alphaMax[3] = {0, 0, 0}, nAct = 0, nBand = 0;
  // StencilLLF: HRLE key and finalAlphas of this thread's last passing call
  unsigned long long lastKey = 0;
  T lastAlpha[3] = {0, 0, 0};
  // batching form: the domain whose partial reductions the registers hold;
  // they go to its RED_* words when the warp moves to another domain's brick
  int dom = -1;
  double delta = A.g.delta;
  const auto flushDomain = [&] {
    minBits = warpMinU64(minBits);
    for (int d = 0; d < 3; ++d) alphaMax[d] = warpMaxU64(alphaMax[d]);
    for (int o = 16; o > 0; o >>= 1) nAct += __shfl_xor_sync(0xffffffffu, nAct, o);
    if (lane == 0) {
      unsigned long long *red = A.domRed + (size_t)RED_WORDS * dom;
      if (MODE == 0 && minBits != ~0ull) atomicMin(red + RED_MIN, minBits);
      for (int d = 0; d < 3; ++d)
        if (alphaMax[d]) atomicMax(red + RED_ALPHA + d, alphaMax[d]);
      if (MODE == 0 && nAct) atomicAdd(red + RED_ACTIVE, nAct);
    }
    minBits = ~0ull, alphaMax[0] = alphaMax[1] = alphaMax[2] = 0, nAct = nBand = 0;
  };
  for (int w = warp; w < n; w += nWarps) {
    const int slot = A.slotList[w];
    if constexpr (BATCH) {
      const int d = A.slotDom[slot];
      if (d != dom) {
        if (dom >= 0) flushDomain();
        dom = d;
        delta = A.domDelta[d];
      }
    }
    const uint64_t own = lane < 8 ? A.def[(size_t)slot * 8 + lane] : 0ull;
    uint64_t a = 0ull;
    if (__any_sync(0xffffffffu, own != 0ull)) a = activePlanes<T>(top.vals, slot);
    int z0 = 0;
    if (A.ownZ) {
      int bx, by, bz;
      brickCoords(A.g, A.m.slotBrick[slot], bx, by, bz);
      z0 = A.g.org[2] + bz * BS;
    }
    if (lane < 8) {
      if (MODE == 0) A.act[(size_t)slot * 8 + lane] = a;
      const bool planeOwned = !A.ownZ || (z0 + lane >= A.ownLo && z0 + lane < A.ownHi);
      if (planeOwned) {
        nAct += __popcll(a);
        nBand += __popcll(own);
      }
    }
    const int total = listCells(a, list);
    // MODE 0: the brick's entries in the compact rate arrays; a pool that is
    // too small leaves the brick out (the host sees rateNext > rateCap, grows
    // the arrays and runs the pass again)
    unsigned long long rbase = 0;
    if (MODE == 0 && total) {
      if (lane == 0) rbase = atomicAdd(A.rateNext, (unsigned long long)total);
      rbase = __shfl_sync(0xffffffffu, rbase, 0);
      if (rbase + (unsigned long long)total > A.rateCap) {
        if (lane == 0 && A.rateOverflowErr) atomicOr(A.err, A.rateOverflowErr);
        continue;
      }
      if (lane == 0) A.rateBase[slot] = rbase;
    }
    for (int base = 0; base < total; base += 32) {
      const int k = base + lane;
      if (k >= total) continue;
      const int c = list[k];
      const auto vel = [&] {
        if constexpr (TABLE)
          return TableVel{A.velS, A.velV, ((size_t)A.actOff[w] + k) * L * A.velSites,
                          A.velSites, A.alphaTab, ((size_t)A.actOff[w] + k) * L * 81,
                          A.velS2, ((size_t)A.actOff[w] + k) * L * 162};
        else if constexpr (BATCH)
          return FunctorVel{A.domVel[dom]};
        else
          return FunctorVel{desc};
      }();
      const bool owned = !A.ownZ || (z0 + (c >> 6) >= A.ownLo && z0 + (c >> 6) < A.ownHi);
      withStencil<T>(A, slot, c, [&](const auto &S, T value) {
        if constexpr (MODE == 0) {
          constexpr bool STENCIL = FAM == FAM_STENCIL;
          T alphas[STENCIL ? 4 : 3] = {};
          const double step =
              ratePoint<T, std::decay_t<decltype(S)>, std::decay_t<decltype(vel)>, FAM>(
                  A, vel, S, slot, c, value, alphas, delta, (size_t)(rbase + k));
          if (!owned) return; // a ghost point: advanced, not counted
          const unsigned long long sb = stepBits(step);
          minBits = sb < minBits ? sb : minBits;
          if constexpr (STENCIL) {
            if (alphas[3] != T(0)) {
              int bx, by, bz;
              brickCoords(A.g, A.m.slotBrick[slot], bx, by, bz);
              const unsigned long long x = A.g.org[0] + bx * BS + (c & 7) + (1 << 20),
                                       y = A.g.org[1] + by * BS + ((c >> 3) & 7) + (1 << 20),
                                       z = A.g.org[2] + bz * BS + (c >> 6) + (1 << 20);
              const unsigned long long key = (z << 42) | (y << 21) | x;
              if (key > lastKey) {
                lastKey = key;
                for (int d = 0; d < 3; ++d) lastAlpha[d] = alphas[d];
              }
            }
          } else {
            for (int d = 0; d < 3; ++d) {
              const unsigned long long ab = alphaBits((double)alphas[d]);
              alphaMax[d] = ab > alphaMax[d] ? ab : alphaMax[d];
            }
          }
        } else {
        for (int lower = 0; lower < L; ++lower) {
          const T lv = lower == L - 1 ? value : lsValueAt<T>(A.ls[lower], slot, c);
          if ((double)lv <= (double)value + 1e-4) {
            T normal[3];
            T normalModulus = 0.;
            for (int d = 0; d < 3; ++d) {
              const T phiPos = S.axis(d, 1);
              const T phiNeg = S.axis(d, -1);
              normal[d] = phiPos - phiNeg;
              normalModulus += normal[d] * normal[d];
            }
            normalModulus = T(1.) / sqrt(normalModulus);
            for (int d = 0; d < 3; ++d) normal[d] *= normalModulus;
            T scaVel, vecVel[3];
            vel.get(lower, normal, 0, scaVel, vecVel);
            if (owned)
              for (int d = 0; d < 3; ++d) {
                const unsigned long long ab =
                    alphaBits((double)fabs((scaVel + vecVel[d]) * normal[d]));
                alphaMax[d] = ab > alphaMax[d] ? ab : alphaMax[d];
              }
            break;
          }
        }
        }
      });
    }
  }
  if constexpr (FAM == FAM_STENCIL && MODE == 0) {
    const unsigned long long best = warpMaxU64(lastKey);
    const unsigned owner = __ballot_sync(0xffffffffu, best != 0ull && lastKey == best);
    if (best == 0ull ? lane == 0 : (owner >> lane) & 1u) {
      A.sllfKey[warp] = best;
      for (int d = 0; d < 3; ++d) A.sllfAlpha[3 * warp + d] = (double)lastAlpha[d];
    }
  }
  if constexpr (BATCH) {
    if (dom >= 0) flushDomain();
    return;
  }
  minBits = warpMinU64(minBits);
  for (int d = 0; d < 3; ++d) alphaMax[d] = warpMaxU64(alphaMax[d]);
  for (int o = 16; o > 0; o >>= 1) {
    nAct += __shfl_xor_sync(0xffffffffu, nAct, o);
    nBand += __shfl_xor_sync(0xffffffffu, nBand, o);
  }
  if (lane == 0) {
    if (MODE == 0 && minBits != ~0ull) atomicMin(A.minStep, minBits);
    if (A.alphaMax)
      for (int d = 0; d < 3; ++d)
        if (alphaMax[d]) atomicMax(&A.alphaMax[d], alphaMax[d]);
    if (MODE == 0 && A.counts) {
      if (nAct) atomicAdd(&A.counts[0], nAct);
      if (nBand) atomicAdd(&A.counts[1], nBand);
    }
  }
}

// StencilLocalLaxFriedrichs time-step alphas: the finalAlphas of the warp
// entry with the largest HRLE key (the last passing call in HRLE order) go to
// alphaOut[0..2] as double bits; nothing is written when no call passed.
__global__ void __launch_bounds__(1024)
    kSllfPick(const unsigned long long *key, const double *alpha, int n,
              unsigned long long *alphaOut) {
  __shared__ unsigned long long sk[32];
  __shared__ int si[32];
  unsigned long long best = 0;
  int bi = -1;
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    if (key[i] > best) best = key[i], bi = i;
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long k2 = __shfl_xor_sync(0xffffffffu, best, o);
    const int i2 = __shfl_xor_sync(0xffffffffu, bi, o);
    if (k2 > best) best = k2, bi = i2;
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sk[wid] = best, si[wid] = bi;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
      if (sk[w] > best) best = sk[w], bi = si[w];
    if (best != 0ull && bi >= 0)
      for (int d = 0; d < 3; ++d) alphaOut[d] = (unsigned long long)__double_as_longlong(alpha[3 * bi + d]);
  }
}

// Value update of updateLevelSet (lsAdvect.hpp:725-777) for every active
// point, in place on the top level set (the Reduce(1) part is applied by the
// rebuild pass that follows).
// `lo` (FP32 top level set with a compensation term, else null): the value is
// hi + lo, the update and the stop-chain walk run in double and the result is
// split into hi and lo again.
// pvel/pdiss (setSaveAdvectionVelocities, else null): each updated point's
// last leg rate (time x velocity) and the dissipation of the chain entry it
// ended on (rateD), lsAdvect.hpp:764-767.
template <class T>
__global__ void __launch_bounds__(RATE_THREADS)
    kUpdate(const int *slotList, const int *nSlots, const uint64_t *act, T *vals,
            const T *rateV, const T *rateStop, const uint8_t *rateLen,
            const unsigned long long *rateBase, size_t rateCap, int L,
            double dt, int *err, float *lo, T *pvel, T *pdiss, const T *rateD,
            const int *slotDom = nullptr, const double *domDt = nullptr) {
  __shared__ uint16_t sList[RATE_THREADS / 32][BV];
  uint16_t *list = sList[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nWarps = (gridDim.x * blockDim.x) >> 5;
  const int n = *nSlots;
  for (int w = warp; w < n; w += nWarps) {
    const int slot = slotList[w];
    const uint64_t a = lane < 8 ? act[(size_t)slot * 8 + lane] : 0ull;
    if (!__any_sync(0xffffffffu, a != 0ull)) continue;
    // batching form: the time step of the slot's domain
    const double dtS = domDt ? domDt[slotDom[slot]] : dt;
    const int total = listCells(a, list);
    const unsigned long long rbase = rateBase[slot];
    for (int base = 0; base < total; base += 32) {
      const int k = base + lane;
      if (k >= total) continue;
      const int c = list[k];
      const size_t q = (size_t)slot * BV + c;
      const size_t r = (size_t)(rbase + k); // this point's rate entries
      if (r >= rateCap) { // the rate pass left this brick out (storage too small)
        atomicOr(err, 1024);
        continue;
      }
      int len = rateLen[r];
      if (len < 1 || len > L) {
        atomicOr(err, 2);
        len = 1;
      }
      if constexpr (sizeof(T) == 4) {
        if (lo) {
          double value = withLo((double)vals[q], lo[q]);
          double time = dtS;
          int j = 0;
          double velocity = rateV[r];
          double rate = time * velocity;
          while (fabs((double)rateStop[(size_t)j * rateCap + r] - value) < fabs(rate)) {
            const double stop = rateStop[(size_t)j * rateCap + r];
            time -= fabs((stop - value) / velocity);
            value = stop;
            ++j;
            if (j >= len) {
              atomicOr(err, 2);
              break;
            }
            velocity = rateV[(size_t)j * rateCap + r];
            rate = time * velocity;
          }
          value -= rate;
          const float hi = (float)value;
          vals[q] = hi;
          lo[q] = (float)(value - (double)hi);
          if (pvel) {
            const int jj = j < len ? j : len - 1; // j == len only after a chain overrun
            pvel[q] = T(rate), pdiss[q] = rateD[(size_t)jj * rateCap + r];
          }
          continue;
        }
      }
      T value = vals[q];
      double time = dtS;
      int j = 0;
      T velocity = rateV[r];
      T rate = T(time * velocity);
      while (fabs(rateStop[(size_t)j * rateCap + r] - value) < fabs(rate)) {
        const T stop = rateStop[(size_t)j * rateCap + r];
        time -= fabs((stop - value) / velocity);
        value = stop;
        ++j;
        if (j >= len) {
          atomicOr(err, 2);
          break;
        }
        velocity = rateV[(size_t)j * rateCap + r];
        rate = T(time * velocity);
      }
      value -= rate;
      vals[q] = value;
      if (pvel) {
        const int jj = j < len ? j : len - 1; // j == len only after a chain overrun
        pvel[q] = rate, pdiss[q] = rateD[(size_t)jj * rateCap + r];
      }
    }
  }
}

} // namespace
} // namespace vlsg
