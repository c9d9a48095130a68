// vlsg_compare.cuh -- the comparison of two level sets' exchange arrays
// (point sets, values, zero-crossing nodes) on the device; see
// vlsg_metrics.cuh for the rules.  Independent of the storage type.
#pragma once

#include <cstdint>

#include "vlsg_common.cuh"

namespace vlsg {
namespace { // internal linkage: every compilation unit has its own copy

__device__ inline uint64_t cellKeyOf(int x, int y, int z) {
  const uint64_t off = 1ull << 20;
  return ((uint64_t)(z + (int)off) << 42) | ((uint64_t)(y + (int)off) << 21) |
         (uint64_t)(x + (int)off);
}

__device__ inline uint64_t keyOf(const int32_t *idx, int64_t i) {
  return cellKeyOf(idx[3 * i], idx[3 * i + 1], idx[3 * i + 2]);
}

// Keys of an exchange point list (HRLE order == ascending key order).
__global__ void kPointKeys(const int32_t *idx, int64_t n, uint64_t *keys) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    keys[i] = keyOf(idx, i);
}

__device__ inline int64_t findKey(const uint64_t *keys, int64_t n, uint64_t k) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (keys[mid] < k) lo = mid + 1;
    else hi = mid;
  }
  return (lo < n && keys[lo] == k) ? lo : -1;
}

// Accumulators of a comparison (device).
struct CompareAcc {
  unsigned long long onlyDefined; // defined here, not in the other
  unsigned long long onlyActive;  // active here, not active in the other
  unsigned long long active;      // active points here
  unsigned long long common;      // points defined in both (counted from A)
  unsigned long long maxDiff;     // bits of max |a - b|
  double sumSq;                   // sum of (a - b)^2
  unsigned long long above[4];    // |a - b| above 1e-6, 1e-5, 1e-4, 1e-3
};

// Points of `a` against the sorted keys of `b`.
__global__ void kComparePoints(const uint64_t *ka, const double *va, int64_t na,
                               const uint64_t *kb, const double *vb, int64_t nb, int countCommon,
                               CompareAcc *acc) {
  unsigned long long onlyDef = 0, onlyAct = 0, act = 0, common = 0, maxBits = 0;
  unsigned long long above[4] = {0, 0, 0, 0};
  double sq = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < na;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double x = va[i];
    const bool ax = fabs(x) <= 0.5;
    act += ax;
    const int64_t j = findKey(kb, nb, ka[i]);
    if (j < 0) {
      ++onlyDef;
      onlyAct += ax;
      continue;
    }
    const double y = vb[j];
    onlyAct += ax && !(fabs(y) <= 0.5);
    if (countCommon) {
      ++common;
      const double d = fabs(x - y);
      const unsigned long long b = orderedBits(d);
      maxBits = b > maxBits ? b : maxBits;
      sq += d * d;
      above[0] += d > 1e-6, above[1] += d > 1e-5, above[2] += d > 1e-4, above[3] += d > 1e-3;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    onlyDef += __shfl_xor_sync(0xffffffffu, onlyDef, o);
    onlyAct += __shfl_xor_sync(0xffffffffu, onlyAct, o);
    act += __shfl_xor_sync(0xffffffffu, act, o);
    common += __shfl_xor_sync(0xffffffffu, common, o);
    const unsigned long long t = __shfl_xor_sync(0xffffffffu, maxBits, o);
    maxBits = t > maxBits ? t : maxBits;
    sq += __shfl_xor_sync(0xffffffffu, sq, o);
    for (int k = 0; k < 4; ++k) above[k] += __shfl_xor_sync(0xffffffffu, above[k], o);
  }
  if ((threadIdx.x & 31) == 0) {
    for (int k = 0; k < 4; ++k)
      if (above[k]) atomicAdd(&acc->above[k], above[k]);
    if (onlyDef) atomicAdd(&acc->onlyDefined, onlyDef);
    if (onlyAct) atomicAdd(&acc->onlyActive, onlyAct);
    if (act) atomicAdd(&acc->active, act);
    if (common) atomicAdd(&acc->common, common);
    if (maxBits) atomicMax(&acc->maxDiff, maxBits);
    if (sq != 0.0) atomicAdd(&acc->sumSq, sq);
  }
}

struct ChamferAcc {
  double sum, sumSq;
  unsigned long long maxBits;
  unsigned long long unresolved; // nearest node farther than the searched shells
};

// Distance (grid units) of every query node to the nearest node of `pts`
// (sorted by cell key); shells of Chebyshev radius 1..4 cells.
__global__ void kNearestNodes(const double *q, int64_t nq, const double *pts,
                              const uint64_t *pkeys, int64_t np, ChamferAcc *acc) {
  double sum = 0, sq = 0;
  unsigned long long maxBits = 0, unresolved = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nq;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double x = q[3 * i], y = q[3 * i + 1], z = q[3 * i + 2];
    const int cx = (int)floor(x), cy = (int)floor(y), cz = (int)floor(z);
    double best = 1e300;
    for (int r = 1; r <= 4; ++r) {
      for (int dz = -r; dz <= r; ++dz)
        for (int dy = -r; dy <= r; ++dy)
          for (int dx = -r; dx <= r; ++dx) {
            const int m = max(abs(dx), max(abs(dy), abs(dz)));
            if (m != r && !(r == 1 && m == 0)) continue; // shell r (r = 1 includes the centre)
            int64_t j = findKey(pkeys, np, cellKeyOf(cx + dx, cy + dy, cz + dz));
            if (j < 0) continue;
            const uint64_t k = pkeys[j];
            for (; j < np && pkeys[j] == k; ++j) {
              const double ex = pts[3 * j] - x, ey = pts[3 * j + 1] - y, ez = pts[3 * j + 2] - z;
              const double d = sqrt(ex * ex + ey * ey + ez * ez);
              best = d < best ? d : best;
            }
          }
      // every node outside shell r is at least r cells away
      if (best <= (double)r) break;
    }
    if (best > 4.0) {
      ++unresolved;
      continue;
    }
    sum += best;
    sq += best * best;
    const unsigned long long b = orderedBits(best);
    maxBits = b > maxBits ? b : maxBits;
  }
  for (int o = 16; o > 0; o >>= 1) {
    sum += __shfl_xor_sync(0xffffffffu, sum, o);
    sq += __shfl_xor_sync(0xffffffffu, sq, o);
    const unsigned long long t = __shfl_xor_sync(0xffffffffu, maxBits, o);
    maxBits = t > maxBits ? t : maxBits;
    unresolved += __shfl_xor_sync(0xffffffffu, unresolved, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (sum != 0.0) atomicAdd(&acc->sum, sum);
    if (sq != 0.0) atomicAdd(&acc->sumSq, sq);
    if (maxBits) atomicMax(&acc->maxBits, maxBits);
    if (unresolved) atomicAdd(&acc->unresolved, unresolved);
  }
}

} // namespace
} // namespace vlsg
