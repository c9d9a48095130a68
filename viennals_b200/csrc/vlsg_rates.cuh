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
// One thread per active point.  Neighbours inside the point's own brick are
// read directly from the slot; the rest go through the brick map.
#pragma once

#include "vlsg_common.cuh"
#include "vlsg_passes.cuh"

namespace vlsg {

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

template <class T> struct RateArgs {
  GridDev g;
  MapView m;
  Buf<T> ls[VLSG_MAX_LEVEL_SETS];
  int L;
  const uint32_t *active;
  const int *nActive;
  int activeCap;
  int scheme;
  double cfl;
  double dissipationAlpha;
  int calcNormals;
  int adaptive;
  double adaptiveFactor;
  int checkDiss;
  T globalAlpha[3];
  // outputs (pool shaped: entry j of cell q at j * poolCells + q)
  T *rateV;
  T *rateStop;
  uint8_t *rateLen;
  size_t poolCells;
  unsigned long long *minStep;  // bits of the smallest non-negative step
  unsigned long long *alphaMax; // bits of the LLF/LLLF alphas
  int *err;
};

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

// Reader of a brick staged in shared memory with a halo of H cells.
template <class T, int H> struct BoxStencil {
  static constexpr int S = BS + 2 * H;
  const T *box;
  int o; // index of the centre cell
  __device__ T at(int dx, int dy, int dz) const { return box[o + (dz * S + dy) * S + dx]; }
  __device__ T axis(int d, int off) const {
    return box[o + off * (d == 0 ? 1 : (d == 1 ? S : S * S))];
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

// One scheme evaluation (Hamiltonian, dissipation) for `material`.
template <class T, class St>
__device__ void evalScheme(const RateArgs<T> &A, const vlsg_velocity_desc &vel,
                           const St &S, T C, int material, T *alphas,
                           T &outG, T &outD) {
  const T gridDelta = T(A.g.delta);
  const int sch = A.scheme;
  if (sch == VLSG_WENO_3RD_ORDER || sch == VLSG_WENO_5TH_ORDER) {
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
    const T sv = scalarVelocity<T>(vel, material, n);
    T vv[3];
    vectorVelocity<T>(vel, material, vv);
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
    const T sv = scalarVelocity<T>(vel, material, n);
    T vv[3];
    vectorVelocity<T>(vel, material, vv);
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
  const T sv = scalarVelocity<T>(vel, material, n);
  T vv[3];
  vectorVelocity<T>(vel, material, vv);
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
  // LocalLaxFriedrichs: alphas over the 3x3x3 box, x fastest
  T alpha[3] = {0, 0, 0};
  for (int q = 0; q < 27; ++q) {
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
    const T scaVel = scalarVelocity<T>(vel, material, normal);
    T vecVel[3];
    vectorVelocity<T>(vel, material, vecVel);
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

template <class T>
__device__ inline T lsValueAt(const Buf<T> &b, int slot, int c) {
  const uint8_t st = b.state[slot];
  if (st == ST_DENSE) return b.vals[(size_t)slot * BV + c];
  return st == ST_UNEG ? Lim<T>::lowest() : Lim<T>::max();
}

// Warp + block reduction of the per-point minima / maxima into global atomics.
__device__ inline void atomicMinStep(unsigned long long *dst, double v) {
  // v >= 0 or NaN; NaN never lowers the minimum (lsAdvect.hpp:591)
  unsigned long long b = (v >= 0.0) ? orderedBits(v + 0.0) : ~0ull;
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long t = __shfl_xor_sync(0xffffffffu, b, o);
    b = t < b ? t : b;
  }
  if ((threadIdx.x & 31) == 0 && b != ~0ull) atomicMin(dst, b);
}
__device__ inline void atomicMaxAlpha(unsigned long long *dst, double v) {
  unsigned long long b = (v > 0.0) ? orderedBits(v) : 0ull;
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long t = __shfl_xor_sync(0xffffffffu, b, o);
    b = t > b ? t : b;
  }
  if ((threadIdx.x & 31) == 0 && b != 0ull) atomicMax(dst, b);
}

// integrateTime for one active point (lsAdvect.hpp:501-592): the material
// chain, the stored rates (velocity as updateLevelSet applies it,
// lsAdvect.hpp:738-744, and the stop value) and the point's time budget.
template <class T, class St>
__device__ inline double ratePoint(const RateArgs<T> &A, const vlsg_velocity_desc &vel,
                                   const St &S, int slot, int c, T C, T *alphas) {
  const int L = A.L;
  const size_t q = (size_t)slot * BV + c;
  T value = C;
  double maxStepTime = 0;
  double cfl = A.cfl;
  int len = 0;
  for (int cur = L - 1; cur >= 0; --cur) {
    T g = 0, d = 0;
    for (int lower = 0; lower < L; ++lower) {
      const T lv = lower == L - 1 ? C : lsValueAt<T>(A.ls[lower], slot, c);
      if ((double)lv <= (double)value + 1e-4) {
        evalScheme<T>(A, vel, S, C, lower, alphas, g, d);
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
    A.rateV[(size_t)len * A.poolCells + q] = veff;
    A.rateStop[(size_t)len * A.poolCells + q] = stop;
    ++len;
    if (done) break;
  }
  A.rateLen[q] = (uint8_t)len;
  return maxStepTime;
}

template <class T>
__global__ void __launch_bounds__(RATE_THREADS)
    kRates(RateArgs<T> A, const vlsg_velocity_desc vel) {
  const int n = min(*A.nActive, A.activeCap);
  const int L = A.L;
  const Buf<T> &top = A.ls[L - 1];
  for (int base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    const int i = base + threadIdx.x;
    double maxStepTime = -1.0; // "no point"
    T alphas[3] = {0, 0, 0};
    if (i < n) {
      const uint32_t q = A.active[i];
      const int slot = q >> 9, c = q & 511;
      const int bi = A.m.slotBrick[slot];
      int bx, by, bz;
      brickCoords(A.g, bi, bx, by, bz);
      const Stencil<T> S{A.g, A.m, top, slot, c & 7, (c >> 3) & 7, c >> 6,
                         A.g.org[0] + bx * BS, A.g.org[1] + by * BS,
                         A.g.org[2] + bz * BS};
      const T C = top.vals[(size_t)slot * BV + c];
      maxStepTime = ratePoint<T>(A, vel, S, slot, c, C, alphas);
    }
    atomicMinStep(A.minStep, maxStepTime);
    if (A.alphaMax) {
      for (int k = 0; k < 3; ++k) atomicMaxAlpha(&A.alphaMax[k], (double)alphas[k]);
    }
  }
}

// findGlobalAlphas, lsAdvect.hpp:90-195.
template <class T>
__global__ void __launch_bounds__(RATE_THREADS)
    kGlobalAlphas(RateArgs<T> A, const vlsg_velocity_desc vel) {
  const int n = min(*A.nActive, A.activeCap);
  const int L = A.L;
  const Buf<T> &top = A.ls[L - 1];
  for (int base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    const int i = base + threadIdx.x;
    T la[3] = {0, 0, 0};
    if (i < n) {
      const uint32_t q = A.active[i];
      const int slot = q >> 9, c = q & 511;
      const int bi = A.m.slotBrick[slot];
      int bx, by, bz;
      brickCoords(A.g, bi, bx, by, bz);
      const Stencil<T> S{A.g, A.m, top, slot, c & 7, (c >> 3) & 7, c >> 6,
                         A.g.org[0] + bx * BS, A.g.org[1] + by * BS,
                         A.g.org[2] + bz * BS};
      const T value = top.vals[(size_t)slot * BV + c];
      for (int lower = 0; lower < L; ++lower) {
        const T lv = lower == L - 1 ? value : lsValueAt<T>(A.ls[lower], slot, c);
        if ((double)lv <= (double)value + 1e-4) {
          T normal[3];
          T normalModulus = 0.;
          for (int k = 0; k < 3; ++k) {
            const T phiPos = S.axis(k, 1);
            const T phiNeg = S.axis(k, -1);
            normal[k] = phiPos - phiNeg;
            normalModulus += normal[k] * normal[k];
          }
          normalModulus = T(1.) / sqrt(normalModulus);
          for (int k = 0; k < 3; ++k) normal[k] *= normalModulus;
          const T scaVel = scalarVelocity<T>(vel, lower, normal);
          T vecVel[3];
          vectorVelocity<T>(vel, lower, vecVel);
          for (int k = 0; k < 3; ++k) {
            const T tempAlpha = fabs((scaVel + vecVel[k]) * normal[k]);
            la[k] = stdMax(la[k], tempAlpha);
          }
          break;
        }
      }
    }
    for (int k = 0; k < 3; ++k) atomicMaxAlpha(&A.alphaMax[k], (double)la[k]);
  }
}

// Reduce(1) + value update of updateLevelSet, in place on the top level set.
template <class T> struct UpdateArgs {
  GridDev g;
  MapView m;
  const int *slotList;
  const int *nSlots;
  T *vals;
  uint8_t *state;
  uint8_t *hasDef;
  const T *rateV;
  const T *rateStop;
  const uint8_t *rateLen;
  size_t poolCells;
  int L;
  double dt;
  int *err;
  unsigned long long *defCount;
};

template <class T>
__global__ void __launch_bounds__(RATE_THREADS) kUpdate(UpdateArgs<T> U) {
  const int n = *U.nSlots;
  for (int it = blockIdx.x; it < n; it += gridDim.x) {
    const int slot = U.slotList[it];
    const uint8_t st = U.state[slot];
    if (st != ST_DENSE) continue; // uniform: Reduce keeps it as it is
    const int bi = U.m.slotBrick[slot];
    int bx, by, bz;
    brickCoords(U.g, bi, bx, by, bz);
    T res[2];
    bool anyDef = false, allPos = true, allNeg = true;
    for (int k = 0; k < 2; ++k) {
      const int c = threadIdx.x + k * RATE_THREADS;
      const size_t q = (size_t)slot * BV + c;
      T value = U.vals[q];
      if (isDef(value) && fabs(value) <= T(0.5)) {
        int len = U.rateLen[q];
        if (len < 1 || len > U.L) {
          atomicOr(U.err, 2);
          len = 1;
        }
        double time = U.dt;
        int j = 0;
        T velocity = U.rateV[q];
        T rate = T(time * velocity);
        while (fabs(U.rateStop[(size_t)j * U.poolCells + q] - value) < fabs(rate)) {
          const T stop = U.rateStop[(size_t)j * U.poolCells + q];
          time -= fabs((stop - value) / velocity);
          value = stop;
          ++j;
          if (j >= len) {
            atomicOr(U.err, 2);
            break;
          }
          velocity = U.rateV[(size_t)j * U.poolCells + q];
          rate = T(time * velocity);
        }
        value -= rate;
      } else {
        value = value < 0 ? Lim<T>::lowest() : Lim<T>::max();
      }
      const int lx = c & 7, ly = (c >> 3) & 7, lz = c >> 6;
      if (!cellExists(U.g, U.g.org[0] + bx * BS + lx, U.g.org[1] + by * BS + ly,
                      U.g.org[2] + bz * BS + lz))
        value = Lim<T>::max();
      else if (isDef(value)) anyDef = true;
      else if (value < 0) allPos = false;
      else allNeg = false;
      res[k] = value;
    }
    countDefined<T>(res, U.defCount);
    const int any = __syncthreads_or(anyDef);
    const int ap = __syncthreads_and(allPos);
    const int an = __syncthreads_and(allNeg);
    if (!any && (ap || an)) {
      if (threadIdx.x == 0) {
        U.state[slot] = ap ? ST_UPOS : ST_UNEG;
        U.hasDef[slot] = 0;
      }
    } else {
      for (int k = 0; k < 2; ++k) U.vals[(size_t)slot * BV + threadIdx.x + k * RATE_THREADS] = res[k];
      if (threadIdx.x == 0) U.hasDef[slot] = any ? 1 : 0;
    }
    __syncthreads();
  }
}

// Compact the active points (defined, |phi| <= 0.5) of the top level set.
template <class T>
__global__ void __launch_bounds__(RATE_THREADS)
    kCompactActive(const int *slotList, const int *nSlots, Buf<T> top,
                   uint32_t *active, int *nActive, int activeCap, int *err,
                   unsigned long long *bandCount) {
  const int n = *nSlots;
  for (int it = blockIdx.x; it < n; it += gridDim.x) {
    const int slot = slotList[it];
    if (top.state[slot] != ST_DENSE) continue;
    for (int k = 0; k < 2; ++k) {
      const int c = threadIdx.x + k * RATE_THREADS;
      const T v = top.vals[(size_t)slot * BV + c];
      const bool act = isDef(v) && fabs(v) <= T(0.5);
      const int nd = __syncthreads_count(isDef(v));
      if (threadIdx.x == 0 && nd) atomicAdd(bandCount, (unsigned long long)nd);
      const unsigned mask = __ballot_sync(0xffffffffu, act);
      const int lane = threadIdx.x & 31;
      int base = 0;
      if (lane == 0 && mask) base = atomicAdd(nActive, __popc(mask));
      base = __shfl_sync(0xffffffffu, base, 0);
      const int pos = base + __popc(mask & ((1u << lane) - 1));
      if (act) {
        if (pos < activeCap) active[pos] = ((uint32_t)slot << 9) | c;
        else atomicOr(err, 16);
      }
    }
  }
}

} // namespace vlsg
