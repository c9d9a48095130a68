// vlsg_velcb.cuh -- host velocity callbacks (viennals::VelocityField with
// user code, lsVelocityField.hpp:17-30).
//
// Before a rate kernel runs in callback mode, kVelGather writes one query per
// active point, material and evaluation site: the coordinate (index *
// gridDelta), the material, the normal the scheme hands the velocity field
// there and the point id -- the rank of the point among the defined points of
// the (expanded) top level set in HRLE order, what
// neighborIterator.getCenter().getPointId() returns in the reference
// (e.g. lsWENO.hpp:132-137).  The host answers the queries through the
// callback, and the rate kernel reads the answers (TableVel) where the device
// functor would be evaluated.  Every material is asked for every point (the
// reference asks only the materials its chain walk reaches, and the box
// neighbours of LocalLaxFriedrichs only when the gradient term is non-zero):
// the same values for any velocity field that is a function of its
// arguments.
//
// The normals restate, expression for expression, the ones evalScheme and
// kRates<.., 1> compute (lsWENO.hpp:113-129, lsEngquistOsher.hpp:124-138,
// lsLaxFriedrichs.hpp / lsLocalLaxFriedrichs.hpp / lsLocalLocalLaxFriedrichs.hpp
// central normals, lsLocalLaxFriedrichs.hpp:194-212 for the box, and
// lsAdvect.hpp:155-166 for findGlobalAlphas).
#pragma once

#include "vlsg_exchange.cuh"
#include "vlsg_frontier.cuh"
#include "vlsg_rates.cuh"

namespace vlsg {
namespace { // internal linkage: every compilation unit has its own copy

// Evaluation sites per point: LocalLaxFriedrichs also asks its 27 box
// neighbours (site 1 + q, x fastest) in the rate pass.
// StencilLocalLaxFriedrichs asks its 27 stencil points (site 1 + q) in a
// first round and the nudged normals (kStencilGather) in a second.
inline int velocitySites(int scheme, int mode) {
  return (mode == 0 && (scheme == VLSG_LOCAL_LAX_FRIEDRICHS_1ST_ORDER ||
                        scheme == VLSG_LOCAL_LAX_FRIEDRICHS_2ND_ORDER ||
                        scheme == VLSG_STENCIL_LOCAL_LAX_FRIEDRICHS_1ST_ORDER))
             ? 28
             : 1;
}

// The normal the scheme passes to the velocity field at the point itself.
template <class T, class St>
__device__ inline void centreNormal(const RateArgs<T> &A, const St &S, T C, T n[3]) {
  const int sch = A.scheme;
  n[0] = n[1] = n[2] = T(0);
  if (sch == VLSG_STENCIL_LOCAL_LAX_FRIEDRICHS_1ST_ORDER) {
    sllfNormal<T>(S, A.g.delta, 0, 0, 0, n);
    return;
  }
  if (sch == VLSG_WENO_3RD_ORDER || sch == VLSG_WENO_5TH_ORDER) {
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
    return;
  }
  if (sch == VLSG_ENGQUIST_OSHER_1ST_ORDER || sch == VLSG_ENGQUIST_OSHER_2ND_ORDER) {
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
    return;
  }
  const int order = (sch == VLSG_LAX_FRIEDRICHS_2ND_ORDER ||
                     sch == VLSG_LOCAL_LOCAL_LAX_FRIEDRICHS_2ND_ORDER ||
                     sch == VLSG_LOCAL_LAX_FRIEDRICHS_2ND_ORDER)
                        ? 2
                        : 1;
  const bool globalLF = (sch == VLSG_LAX_FRIEDRICHS_1ST_ORDER ||
                         sch == VLSG_LAX_FRIEDRICHS_2ND_ORDER);
  const bool calcNormal = globalLF ? (A.calcNormals != 0) : true;
  if (!calcNormal) return;
  const T gridDelta = T(A.g.delta);
  T normalModulus = 0;
  for (int i = 0; i < 3; i++) {
    T diffPos, diffNeg;
    oneSided<T>(S, i, C, gridDelta, order, diffPos, diffNeg);
    n[i] = (diffNeg + diffPos) * T(0.5);
    normalModulus += n[i] * n[i];
  }
  normalModulus = T(1.) / sqrt(normalModulus);
  for (int i = 0; i < 3; ++i) n[i] *= normalModulus;
}

// The normal LocalLaxFriedrichs passes for box neighbour q.
template <class T, class St>
__device__ inline void boxNormal(const St &S, T gridDelta, int q, T normal[3]) {
  const int ox = q % 3 - 1, oy = (q / 3) % 3 - 1, oz = q / 9 - 1;
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
}

// The normal findGlobalAlphas passes.
template <class T, class St> __device__ inline void alphaNormal(const St &S, T normal[3]) {
  T normalModulus = 0.;
  for (int d = 0; d < 3; ++d) {
    const T phiPos = S.axis(d, 1);
    const T phiNeg = S.axis(d, -1);
    normal[d] = phiPos - phiNeg;
    normalModulus += normal[d] * normal[d];
  }
  normalModulus = T(1.) / sqrt(normalModulus);
  for (int d = 0; d < 3; ++d) normal[d] *= normalModulus;
}

// Active points per slot-list entry (the cells kRates lists).
template <class T> __global__ void __launch_bounds__(RATE_THREADS) kActiveCount(RateArgs<T> A, uint32_t *cnt) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nWarps = (gridDim.x * blockDim.x) >> 5;
  const int n = *A.nSlots;
  const Buf<T> &top = A.ls[A.L - 1];
  for (int w = warp; w < n; w += nWarps) {
    const int slot = A.slotList[w];
    const uint64_t own = lane < 8 ? A.def[(size_t)slot * 8 + lane] : 0ull;
    uint64_t a = 0ull;
    if (__any_sync(0xffffffffu, own != 0ull)) a = activePlanes<T>(top.vals, slot);
    int c = lane < 8 ? __popcll(a) : 0;
    for (int o = 4; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0) cnt[w] = (uint32_t)c;
  }
}

// Point ids of the defined cells of one buffer: the exchange's segment
// offsets (pos: ordered index of every allocated brick, bounds: its brick
// row and slab, P: points before every segment).
struct PointRanks {
  const int *slotBrick;
  const uint32_t *pos;
  const int4 *bounds;
  const uint32_t *P;
  const uint64_t *def;
  __device__ uint64_t of(int slot, int c) const {
    const int i = (int)pos[slotBrick[slot]];
    const int lz = c >> 6, ly = (c >> 3) & 7, x = c & 7;
    const unsigned byte = segByte(def, slot, lz, ly);
    return (uint64_t)P[segmentRank(bounds[i], i, lz, ly)] + __popc(byte & ((1u << x) - 1u));
  }
};

// The queries of the rate pass MODE (0: rates, 1: global alphas) for every
// active point p: entry (p * L + material) * sites + site.
template <class T, int MODE>
__global__ void __launch_bounds__(RATE_THREADS)
    kVelGather(RateArgs<T> A, PointRanks R, int sites, double *coord, int32_t *material,
               double *normal, uint64_t *pid) {
  __shared__ uint16_t sList[RATE_THREADS / 32][BV];
  uint16_t *list = sList[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nWarps = (gridDim.x * blockDim.x) >> 5;
  const int n = *A.nSlots;
  const int L = A.L;
  const Buf<T> &top = A.ls[L - 1];
  const double delta = A.g.delta;
  for (int w = warp; w < n; w += nWarps) {
    const int slot = A.slotList[w];
    const uint64_t own = lane < 8 ? A.def[(size_t)slot * 8 + lane] : 0ull;
    uint64_t a = 0ull;
    if (__any_sync(0xffffffffu, own != 0ull)) a = activePlanes<T>(top.vals, slot);
    const int total = listCells(a, list);
    int bx, by, bz;
    brickCoords(A.g, A.m.slotBrick[slot], bx, by, bz);
    for (int k = lane; k < total; k += 32) {
      const int c = list[k];
      const size_t p = (size_t)A.actOff[w] + k;
      const uint64_t id = R.of(slot, c);
      const int idx[3] = {A.g.org[0] + bx * BS + (c & 7), A.g.org[1] + by * BS + ((c >> 3) & 7),
                          A.g.org[2] + bz * BS + (c >> 6)};
      T coordinate[3];
      for (int d = 0; d < 3; ++d) coordinate[d] = T(idx[d] * delta);
      withStencil<T>(A, slot, c, [&](const auto &S, T C) {
        for (int s = 0; s < sites; ++s) {
          T nrm[3], crd[3];
          if (MODE == 1) {
            alphaNormal<T>(S, nrm);
          } else if (s == 0) {
            centreNormal<T>(A, S, C, nrm);
          } else if (A.scheme == VLSG_STENCIL_LOCAL_LAX_FRIEDRICHS_1ST_ORDER) {
            const int q = s - 1;
            sllfNormal<T>(S, delta, q % 3 - 1, (q / 3) % 3 - 1, q / 9 - 1, nrm);
          } else {
            boxNormal<T>(S, T(delta), s - 1, nrm);
          }
          for (int d = 0; d < 3; ++d) crd[d] = coordinate[d];
          if (s > 0) {
            const int off[3] = {(s - 1) % 3 - 1, ((s - 1) / 3) % 3 - 1, (s - 1) / 9 - 1};
            for (int d = 0; d < 3; ++d) crd[d] = T(coordinate[d] + off[d] * delta);
          }
          // D = 2: the box sites above and below the plane are not asked
          // (material -1; the rate kernels read only the plane's)
          const bool unasked = A.g.planar && s > 0 && (s - 1) / 9 != 1;
          for (int m = 0; m < L; ++m) {
            const size_t q = (p * L + m) * sites + s;
            for (int d = 0; d < 3; ++d) {
              coord[3 * q + d] = (double)crd[d];
              normal[3 * q + d] = (double)nrm[d];
            }
            material[q] = unasked ? -1 : m;
            pid[q] = id;
          }
        }
      });
    }
  }
}

// StencilLocalLaxFriedrichs, second round: the nudged normals of every
// active point p, material and stencil point q, built from the first
// round's answers (sites 1 + q) exactly as evalStencilLLF builds them, at
// (p * L + material) * 162 + 6q + 2k (+1 for +DN).
template <class T>
__global__ void __launch_bounds__(RATE_THREADS)
    kStencilGather(RateArgs<T> A, PointRanks R, double *coord, int32_t *material,
                   double *normal, uint64_t *pid) {
  __shared__ uint16_t sList[RATE_THREADS / 32][BV];
  uint16_t *list = sList[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nWarps = (gridDim.x * blockDim.x) >> 5;
  const int n = *A.nSlots;
  const int L = A.L;
  const Buf<T> &top = A.ls[L - 1];
  const double delta = A.g.delta;
  for (int w = warp; w < n; w += nWarps) {
    const int slot = A.slotList[w];
    const uint64_t own = lane < 8 ? A.def[(size_t)slot * 8 + lane] : 0ull;
    uint64_t a = 0ull;
    if (__any_sync(0xffffffffu, own != 0ull)) a = activePlanes<T>(top.vals, slot);
    const int total = listCells(a, list);
    int bx, by, bz;
    brickCoords(A.g, A.m.slotBrick[slot], bx, by, bz);
    for (int k = lane; k < total; k += 32) {
      const int c = list[k];
      const size_t p = (size_t)A.actOff[w] + k;
      const uint64_t id = R.of(slot, c);
      const int idx[3] = {A.g.org[0] + bx * BS + (c & 7), A.g.org[1] + by * BS + ((c >> 3) & 7),
                          A.g.org[2] + bz * BS + (c >> 6)};
      T coordinate[3];
      for (int d = 0; d < 3; ++d) coordinate[d] = T(idx[d] * delta);
      withStencil<T>(A, slot, c, [&](const auto &S, T) {
        for (int q = 0; q < 27; ++q) {
          const int off[3] = {q % 3 - 1, (q / 3) % 3 - 1, q / 9 - 1};
          T ln[3], crd[3];
          sllfNormal<T>(S, delta, off[0], off[1], off[2], ln);
          for (int d = 0; d < 3; ++d) crd[d] = T(coordinate[d] + off[d] * delta);
          for (int m = 0; m < L; ++m) {
            const size_t r1 = (p * L + m) * 28 + 1 + q;
            T lsv = T(A.velS[r1]);
            T lvv[3];
            for (int d = 0; d < 3; ++d) lvv[d] = T(A.velV[3 * r1 + d]);
            for (int dir = 0; dir < 3; ++dir) lsv += lvv[dir] * ln[dir];
            const T DN = sllfEpsilon<T>(lsv, A.sllfEps, delta);
            T np[3] = {ln[0], ln[1], ln[2]}, nn[3] = {ln[0], ln[1], ln[2]};
            for (int kk = 0; kk < 3; ++kk) {
              np[kk] -= DN;
              nn[kk] += DN;
              for (int side = 0; side < 2; ++side) {
                const size_t e = (p * L + m) * 162 + 6 * q + 2 * kk + side;
                const T *nv = side ? nn : np;
                for (int d = 0; d < 3; ++d) {
                  coord[3 * e + d] = (double)crd[d];
                  normal[3 * e + d] = (double)nv[d];
                }
                // D = 2: only the plane's stencil, nudged in x and y, is asked
                material[e] = (A.g.planar && (q / 9 != 1 || kk == 2)) ? -1 : m;
                pid[e] = id;
              }
              np[kk] += DN;
              nn[kk] -= DN;
            }
          }
        }
      });
    }
  }
}

// LocalLaxFriedrichsAnalytical: the alpha queries of every active point p,
// material, box neighbour q and direction, at
// ((p * L + material) * 27 + q) * 3 + dir.
template <class T>
__global__ void __launch_bounds__(RATE_THREADS)
    kAlphaGather(RateArgs<T> A, int32_t *direction, int32_t *material, double *cd) {
  __shared__ uint16_t sList[RATE_THREADS / 32][BV];
  uint16_t *list = sList[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nWarps = (gridDim.x * blockDim.x) >> 5;
  const int n = *A.nSlots;
  const int L = A.L;
  const Buf<T> &top = A.ls[L - 1];
  const T gridDelta = T(A.g.delta);
  for (int w = warp; w < n; w += nWarps) {
    const int slot = A.slotList[w];
    const uint64_t own = lane < 8 ? A.def[(size_t)slot * 8 + lane] : 0ull;
    uint64_t a = 0ull;
    if (__any_sync(0xffffffffu, own != 0ull)) a = activePlanes<T>(top.vals, slot);
    const int total = listCells(a, list);
    for (int k = lane; k < total; k += 32) {
      const int c = list[k];
      const size_t p = (size_t)A.actOff[w] + k;
      withStencil<T>(A, slot, c, [&](const auto &S, T) {
        for (int q = 0; q < 27; ++q) {
          T d3[3];
          boxDifferences<T>(S, gridDelta, q, d3);
          for (int m = 0; m < L; ++m)
            for (int dir = 0; dir < 3; ++dir) {
              const size_t e = ((p * L + m) * 27 + q) * 3 + dir;
              direction[e] = dir;
              material[e] = m;
              for (int k3 = 0; k3 < 3; ++k3) cd[3 * e + k3] = (double)d3[k3];
            }
        }
      });
    }
  }
}

// Point data at the start of an advection: every defined cell of the top
// level set carries its own rank in download order, no saved velocity.
template <class T>
__global__ void kInitPointData(const int *slotList, const int *nSlots, const uint64_t *def,
                               PointRanks R, Payload<T> pd) {
  const size_t n = (size_t)*nSlots * BV;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const int slot = slotList[i / BV];
    const int c = (int)(i % BV);
    if (!((def[(size_t)slot * 8 + (c >> 6)] >> (c & 63)) & 1ull)) continue;
    const size_t q = (size_t)slot * BV + c;
    pd.src[q] = (int32_t)R.of(slot, c);
    pd.vel[q] = T(0);
    pd.diss[q] = T(0);
  }
}

// Point data of the defined cells in download order (the exchange layout of
// kSegScatter: segment offsets P, x order within a segment).
template <class T>
__global__ void kSegPointData(const int *ob, int nAlloc, const int *brickMap, const int4 *bounds,
                              const uint64_t *def, const uint32_t *P, Payload<T> pd,
                              int64_t *srcOut, double *velOut, double *dissOut) {
  const size_t nSeg = (size_t)nAlloc * 64;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < nSeg;
       e += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(e >> 6), lz = (int)(e >> 3) & 7, ly = (int)e & 7;
    const int slot = brickMap[ob[i]];
    const unsigned byte = segByte(def, slot, lz, ly);
    if (!byte) continue;
    uint32_t pos = P[segmentRank(bounds[i], i, lz, ly)];
    for (unsigned m = byte; m; m &= m - 1) {
      const size_t q = (size_t)slot * BV + lz * 64 + ly * 8 + (__ffs(m) - 1);
      srcOut[pos] = pd.src[q];
      velOut[pos] = (double)pd.vel[q];
      dissOut[pos] = (double)pd.diss[q];
      ++pos;
    }
  }
}

} // namespace
} // namespace vlsg
