// vlsg_fused.cuh -- temporally blocked band passes over a brick neighbour
// table.
//
// On "brick-aligned" domains (every bounded direction periodic with a
// multiple of 8 points; infinite directions anywhere) a cell's star
// neighbours always lie in the 3x3x3 bricks around its own, so every slot
// keeps a table of its 27 neighbour bricks (slot, or -1-brick for an
// unallocated one) and a pass stages the brick plus a halo of R cells in
// shared memory in one go.  R consecutive star passes (Expand cycles,
// lsExpand.hpp:62-169) then run on the staged box -- each cycle one cell
// narrower -- and only the centre brick is written: one sweep of the pool
// instead of R.  The result is identical to R separate passes: every cycle
// evaluates exactly the same rule on exactly the same neighbour values.
//
// The same staging runs the per-point update of updateLevelSet
// (lsAdvect.hpp:725-777, including Reduce(1), lsReduce.hpp:281-296) on the
// cells it loads and the rebuild rule (lsAdvect.hpp:299-415) on the result,
// fusing update + rebuild into one sweep.
#pragma once

#include "vlsg_passes.cuh"
#include "vlsg_rates.cuh"

namespace vlsg {

constexpr int FUSED_THREADS = 256;
constexpr int MAX_FUSED_CYCLES = 4;

// 27-neighbour table of every listed slot (k = (dz+1)*9 + (dy+1)*3 + dx+1).
__global__ void kBuildNeighbours(GridDev g, const int *brickMap, const int *slotBrick,
                                 const int *slotList, const int *nSlots, int *nbr) {
  const int n = *nSlots;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int slot = slotList[i];
    int bx, by, bz;
    brickCoords(g, slotBrick[slot], bx, by, bz);
    for (int k = 0; k < 27; ++k) {
      int c[3] = {bx + k % 3 - 1, by + (k / 3) % 3 - 1, bz + k / 9 - 1};
      bool outside = false;
      for (int d = 0; d < 3; ++d) {
        if (c[d] >= 0 && c[d] < g.nb[d]) continue;
        if (g.bc[d] == VLSG_PERIODIC_BOUNDARY) {
          c[d] = (c[d] + g.nb[d]) % g.nb[d];
        } else {
          // outside the box (infinite direction): far region of the
          // nearest box brick
          c[d] = c[d] < 0 ? 0 : g.nb[d] - 1;
          outside = true;
        }
      }
      const int bi = brickIndex(g, c[0], c[1], c[2]);
      const int s = brickMap[bi];
      nbr[(size_t)slot * 27 + k] = (s >= 0 && !outside) ? s : -1 - bi;
    }
  }
}

template <class T>
__device__ inline T nbrCell(const Buf<T> &b, int ref, int local) {
  if (ref < 0) return b.farSign[-1 - ref] < 0 ? Lim<T>::lowest() : Lim<T>::max();
  const uint8_t st = b.state[ref];
  if (st == ST_DENSE) return b.vals[(size_t)ref * BV + local];
  return st == ST_UNEG ? Lim<T>::lowest() : Lim<T>::max();
}

// Sign (+-1) of a uniform neighbour, 0 when it is dense.
template <class T> __device__ inline int nbrUniformSign(const Buf<T> &b, int ref) {
  if (ref < 0) return b.farSign[-1 - ref] < 0 ? -1 : 1;
  const uint8_t st = b.state[ref];
  if (st == ST_DENSE) return 0;
  return st == ST_UNEG ? -1 : 1;
}

// Slots whose output can differ from their input: dense ones, and uniform
// ones next to a dense (or differently signed) brick.  The others keep their
// state (written here, since states are double buffered).
template <class T>
__global__ void kBuildWork(const int *slotList, const int *nSlots, const int *nbr, Buf<T> in,
                           uint8_t *outState, uint8_t *hasDef, int *work, int *nWork) {
  const int n = *nSlots;
  for (int base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    const int i = base + threadIdx.x;
    bool need = false;
    int slot = -1;
    if (i < n) {
      slot = slotList[i];
      const uint8_t st = in.state[slot];
      if (st == ST_DENSE) {
        need = true;
      } else {
        const int s = st == ST_UNEG ? -1 : 1;
        for (int k = 0; k < 27 && !need; ++k)
          if (nbrUniformSign<T>(in, nbr[(size_t)slot * 27 + k]) != s) need = true;
        if (!need) {
          outState[slot] = st;
          hasDef[slot] = 0;
        }
      }
    }
    const unsigned mask = __ballot_sync(0xffffffffu, need);
    const int lane = threadIdx.x & 31;
    int off = 0;
    if (lane == 0 && mask) off = atomicAdd(nWork, __popc(mask));
    off = __shfl_sync(0xffffffffu, off, 0);
    if (need) work[off + __popc(mask & ((1u << lane) - 1))] = slot;
  }
}

// Stage brick `slot` with a halo of H cells: box[(z+H)*S*S + (y+H)*S + x+H],
// S = 8 + 2H, coordinates in [-H, 8+H).
template <class T, int H, class Load>
__device__ inline void stageBox(T *box, const int *nb27, Load load) {
  constexpr int S = BS + 2 * H;
  for (int q = threadIdx.x; q < S * S * S; q += blockDim.x) {
    const int x = q % S - H, y = (q / S) % S - H, z = q / (S * S) - H;
    const int kx = x < 0 ? 0 : (x >= BS ? 2 : 1);
    const int ky = y < 0 ? 0 : (y >= BS ? 2 : 1);
    const int kz = z < 0 ? 0 : (z >= BS ? 2 : 1);
    const int k = kz * 9 + ky * 3 + kx;
    const int local = ((z + BS) & 7) * 64 + ((y + BS) & 7) * 8 + ((x + BS) & 7);
    box[q] = load(k, nb27[k], local);
  }
}

// Neighbour refs of a slot and, per neighbour, the sentinel its cells take
// when it is not dense (0 = dense: read the cell).
template <class T> struct NbrCache {
  int ref[27];
  T fill[27];
  __device__ void load(const int *nbr, int slot, const Buf<T> &b) {
    if (threadIdx.x < 27) {
      const int r = nbr[(size_t)slot * 27 + threadIdx.x];
      ref[threadIdx.x] = r;
      T f;
      if (r < 0) {
        f = b.farSign[-1 - r] < 0 ? Lim<T>::lowest() : Lim<T>::max();
      } else {
        const uint8_t st = b.state[r];
        f = st == ST_DENSE ? T(0) : (st == ST_UNEG ? Lim<T>::lowest() : Lim<T>::max());
      }
      fill[threadIdx.x] = f;
    }
  }
  __device__ T cell(const Buf<T> &b, int k, int local) const {
    const T f = fill[k];
    return f == T(0) ? b.vals[(size_t)ref[k] * BV + local] : f;
  }
};

template <class T> struct ExpandCycles {
  int n;                       // cycles in this launch (<= MAX_FUSED_CYCLES)
  T totalLimit;
  T limit[MAX_FUSED_CYCLES];
};

// `R` Expand cycles in one sweep.
template <class T, int R>
__global__ void __launch_bounds__(FUSED_THREADS)
    kExpandFused(GridDev g, const int *work, const int *nWork, const int *nbr, Buf<T> in,
                 PassOut<T> out, ExpandCycles<T> cyc) {
  constexpr int S = BS + 2 * R;
  extern __shared__ unsigned char smem_raw[];
  T *boxA = reinterpret_cast<T *>(smem_raw);
  T *boxB = boxA + S * S * S;
  __shared__ NbrCache<T> nc;
  const int n = *nWork;
  for (int it = blockIdx.x; it < n; it += gridDim.x) {
    const int slot = work[it];
    nc.load(nbr, slot, in);
    __syncthreads();
    stageBox<T, R>(boxA, nc.ref, [&](int k, int, int local) { return nc.cell(in, k, local); });
    __syncthreads();
    T *src = boxA, *dst = boxB;
    for (int c = 0; c < R; ++c) {
      const ExpandRule<T> rule{cyc.totalLimit, cyc.limit[c]};
      const int h = R - 1 - c; // cells still needed around the brick
      const int W = BS + 2 * h;
      for (int q = threadIdx.x; q < W * W * W; q += blockDim.x) {
        const int x = q % W - h, y = (q / W) % W - h, z = q / (W * W) - h;
        const int o = ((z + R) * S + (y + R)) * S + (x + R);
        T nb6[6] = {src[o + 1], src[o + S], src[o + S * S], src[o - 1], src[o - S], src[o - S * S]};
        dst[o] = rule(src[o], nb6);
      }
      __syncthreads();
      T *t = src;
      src = dst;
      dst = t;
    }
    T res[2];
    bool anyDef = false, allPos = true, allNeg = true;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int c = threadIdx.x + k * FUSED_THREADS;
      const int x = c & 7, y = (c >> 3) & 7, z = c >> 6;
      const T o = src[((z + R) * S + (y + R)) * S + (x + R)];
      if (isDef(o)) anyDef = true;
      else if (o < 0) allPos = false;
      else allNeg = false;
      res[k] = o;
    }
    countDefined<T>(res, out.defCount);
    const int any = __syncthreads_or(anyDef);
    const int ap = __syncthreads_and(allPos);
    const int an = __syncthreads_and(allNeg);
    if (!any && (ap || an)) {
      if (threadIdx.x == 0) {
        out.state[slot] = ap ? ST_UPOS : ST_UNEG;
        out.hasDef[slot] = 0;
      }
    } else {
#pragma unroll
      for (int k = 0; k < 2; ++k)
        out.vals[(size_t)slot * BV + threadIdx.x + k * FUSED_THREADS] = res[k];
      if (threadIdx.x == 0) {
        out.state[slot] = ST_DENSE;
        out.hasDef[slot] = any ? 1 : 0;
      }
    }
    __syncthreads();
  }
}

// Width-1 value of one cell after updateLevelSet: the updated value of an
// active point, the Reduce(1) sentinel of any other.
template <class T>
__device__ inline T updatedValue(T value, const T *rateV, const T *rateStop,
                                 const uint8_t *rateLen, size_t poolCells, size_t q, int L,
                                 double dt, int *err) {
  if (!(isDef(value) && fabs(value) <= T(0.5))) return value < 0 ? Lim<T>::lowest() : Lim<T>::max();
  int len = rateLen[q];
  if (len < 1 || len > L) {
    atomicOr(err, 2);
    len = 1;
  }
  double time = dt;
  int j = 0;
  T velocity = rateV[q];
  T rate = T(time * velocity);
  while (fabs(rateStop[(size_t)j * poolCells + q] - value) < fabs(rate)) {
    const T stop = rateStop[(size_t)j * poolCells + q];
    time -= fabs((stop - value) / velocity);
    value = stop;
    ++j;
    if (j >= len) {
      atomicOr(err, 2);
      break;
    }
    velocity = rateV[(size_t)j * poolCells + q];
    rate = T(time * velocity);
  }
  value -= rate;
  return value;
}

// Reduce(1) + update + rebuildLS in one sweep.
template <class T>
__global__ void __launch_bounds__(FUSED_THREADS)
    kUpdateRebuild(GridDev g, const int *work, const int *nWork, const int *nbr, Buf<T> in,
                   PassOut<T> out, const T *rateV, const T *rateStop, const uint8_t *rateLen,
                   size_t poolCells, int L, double dt, double cutoff, int *err) {
  constexpr int S = BS + 2;
  __shared__ T box[S * S * S];
  __shared__ NbrCache<T> nc;
  const int n = *nWork;
  const RebuildRule<T> rule{cutoff};
  for (int it = blockIdx.x; it < n; it += gridDim.x) {
    const int slot = work[it];
    nc.load(nbr, slot, in);
    __syncthreads();
    stageBox<T, 1>(box, nc.ref, [&](int k, int ref, int local) {
      const T v = nc.cell(in, k, local);
      if (nc.fill[k] != T(0)) return v; // not dense: no active point
      return updatedValue<T>(v, rateV, rateStop, rateLen, poolCells,
                             (size_t)ref * BV + local, L, dt, err);
    });
    __syncthreads();
    T res[2];
    bool anyDef = false, allPos = true, allNeg = true;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int c = threadIdx.x + k * FUSED_THREADS;
      const int x = c & 7, y = (c >> 3) & 7, z = c >> 6;
      const int o = ((z + 1) * S + (y + 1)) * S + (x + 1);
      T nb6[6] = {box[o + 1], box[o + S], box[o + S * S], box[o - 1], box[o - S], box[o - S * S]};
      const T r = rule(box[o], nb6);
      if (isDef(r)) anyDef = true;
      else if (r < 0) allPos = false;
      else allNeg = false;
      res[k] = r;
    }
    countDefined<T>(res, out.defCount);
    const int any = __syncthreads_or(anyDef);
    const int ap = __syncthreads_and(allPos);
    const int an = __syncthreads_and(allNeg);
    if (!any && (ap || an)) {
      if (threadIdx.x == 0) {
        out.state[slot] = ap ? ST_UPOS : ST_UNEG;
        out.hasDef[slot] = 0;
      }
    } else {
#pragma unroll
      for (int k = 0; k < 2; ++k)
        out.vals[(size_t)slot * BV + threadIdx.x + k * FUSED_THREADS] = res[k];
      if (threadIdx.x == 0) {
        out.state[slot] = ST_DENSE;
        out.hasDef[slot] = any ? 1 : 0;
      }
    }
    __syncthreads();
  }
}

// Rates of the active points (integrateTime, lsAdvect.hpp:495-593) of every
// dense brick of the top level set: the brick and a halo of 3 cells -- the
// reach of every scheme's stencil (WENO5 star radius 3, the LocalLaxFriedrichs
// 3x3x3 box of normals) -- are staged in shared memory, the brick's active
// cells are collected there and each thread evaluates one active point from
// shared memory.  Also counts the active points and the band cells.
template <class T>
__global__ void __launch_bounds__(FUSED_THREADS)
    kRatesBrick(RateArgs<T> A, const vlsg_velocity_desc vel, const int *slotList,
                const int *nSlots, const int *nbr, int *nActive,
                unsigned long long *bandCount) {
  constexpr int H = 3, S = BS + 2 * H;
  __shared__ T box[S * S * S];
  __shared__ NbrCache<T> nc;
  __shared__ short act[BV];
  __shared__ int nAct;
  const Buf<T> &top = A.ls[A.L - 1];
  const int n = *nSlots;
  for (int it = blockIdx.x; it < n; it += gridDim.x) {
    const int slot = slotList[it];
    if (top.state[slot] != ST_DENSE) continue;
    nc.load(nbr, slot, top);
    if (threadIdx.x == 0) nAct = 0;
    __syncthreads();
    stageBox<T, H>(box, nc.ref, [&](int k, int, int local) { return nc.cell(top, k, local); });
    __syncthreads();
    int nd = 0;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int c = threadIdx.x + k * FUSED_THREADS;
      const T v = box[(((c >> 6) + H) * S + ((c >> 3) & 7) + H) * S + (c & 7) + H];
      nd += __syncthreads_count(isDef(v));
      if (isDef(v) && fabs(v) <= T(0.5)) act[atomicAdd(&nAct, 1)] = (short)c;
    }
    __syncthreads();
    const int na = nAct;
    if (threadIdx.x == 0) {
      if (na) atomicAdd(nActive, na);
      if (nd && bandCount) atomicAdd(bandCount, (unsigned long long)nd);
    }
    const int rounds = (na + FUSED_THREADS - 1) / FUSED_THREADS;
    for (int r = 0; r < rounds; ++r) {
      const int j = r * FUSED_THREADS + threadIdx.x;
      double maxStepTime = -1.0;
      T alphas[3] = {0, 0, 0};
      if (j < na) {
        const int c = act[j];
        const int o = (((c >> 6) + H) * S + ((c >> 3) & 7) + H) * S + (c & 7) + H;
        const BoxStencil<T, H> st{box, o};
        maxStepTime = ratePoint<T>(A, vel, st, slot, c, box[o], alphas);
      }
      atomicMinStep(A.minStep, maxStepTime);
      if (A.alphaMax)
        for (int k = 0; k < 3; ++k) atomicMaxAlpha(&A.alphaMax[k], (double)alphas[k]);
    }
    __syncthreads();
  }
}

// Active points of the top level set, one warp per slot.
template <class T>
__global__ void kCompactActiveWarp(const int *slotList, const int *nSlots, Buf<T> top,
                                   uint32_t *active, int *nActive, int activeCap, int *err,
                                   unsigned long long *bandCount) {
  const int n = *nSlots;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nWarps = (gridDim.x * blockDim.x) >> 5;
  for (int w = warp; w < n; w += nWarps) {
    const int slot = slotList[w];
    if (top.state[slot] != ST_DENSE) continue;
    int nd = 0;
    for (int c0 = 0; c0 < BV; c0 += 32) {
      const int c = c0 + lane;
      const T v = top.vals[(size_t)slot * BV + c];
      const bool act = isDef(v) && fabs(v) <= T(0.5);
      nd += __popc(__ballot_sync(0xffffffffu, isDef(v)));
      const unsigned mask = __ballot_sync(0xffffffffu, act);
      int off = 0;
      if (lane == 0 && mask) off = atomicAdd(nActive, __popc(mask));
      off = __shfl_sync(0xffffffffu, off, 0);
      const int pos = off + __popc(mask & ((1u << lane) - 1));
      if (act) {
        if (pos < activeCap) active[pos] = ((uint32_t)slot << 9) | c;
        else atomicOr(err, 16);
      }
    }
    if (lane == 0 && nd && bandCount) atomicAdd(bandCount, (unsigned long long)nd);
  }
}

// One star pass (Prune, rebuild) staged through the neighbour table.
template <class T, class Rule>
__global__ void __launch_bounds__(FUSED_THREADS)
    kStarTable(const int *work, const int *nWork, const int *nbr, Buf<T> in, PassOut<T> out,
               Rule rule) {
  constexpr int S = BS + 2;
  __shared__ T box[S * S * S];
  __shared__ NbrCache<T> nc;
  const int n = *nWork;
  for (int it = blockIdx.x; it < n; it += gridDim.x) {
    const int slot = work[it];
    nc.load(nbr, slot, in);
    __syncthreads();
    stageBox<T, 1>(box, nc.ref, [&](int k, int, int local) { return nc.cell(in, k, local); });
    __syncthreads();
    T res[2];
    bool anyDef = false, allPos = true, allNeg = true;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int c = threadIdx.x + k * FUSED_THREADS;
      const int x = c & 7, y = (c >> 3) & 7, z = c >> 6;
      const int o = ((z + 1) * S + (y + 1)) * S + (x + 1);
      T nb6[6] = {box[o + 1], box[o + S], box[o + S * S], box[o - 1], box[o - S], box[o - S * S]};
      const T r = rule(box[o], nb6);
      if (isDef(r)) anyDef = true;
      else if (r < 0) allPos = false;
      else allNeg = false;
      res[k] = r;
    }
    countDefined<T>(res, out.defCount);
    const int any = __syncthreads_or(anyDef);
    const int ap = __syncthreads_and(allPos);
    const int an = __syncthreads_and(allNeg);
    if (!any && (ap || an)) {
      if (threadIdx.x == 0) {
        out.state[slot] = ap ? ST_UPOS : ST_UNEG;
        out.hasDef[slot] = 0;
      }
    } else {
#pragma unroll
      for (int k = 0; k < 2; ++k)
        out.vals[(size_t)slot * BV + threadIdx.x + k * FUSED_THREADS] = res[k];
      if (threadIdx.x == 0) {
        out.state[slot] = ST_DENSE;
        out.hasDef[slot] = any ? 1 : 0;
      }
    }
    __syncthreads();
  }
}


} // namespace vlsg
