// vlsg_rows.cuh -- the Expand cycle (lsExpand.hpp:104-157) as a row pass:
// one warp per brick, each lane owns two x-rows of 8 cells.
//
// A lane takes its rows' bytes of the defined masks (the brick's own planes,
// the planes above and below, the face rows of the y and z neighbours and
// the face bits of the x neighbours), dilates them with shifts and ORs, and
// evaluates ExpandRule directly on the candidate bits of its rows: no cell
// list, no shared memory and no per-brick ballots beyond the publication of
// the new masks.  The rule reads old values only; changes go to the warp's
// change-log segment like every other pass (vlsg_frontier.cuh).  Bricks next
// to a boundary that remaps cells keep the generic per-candidate path.
#pragma once

#include "vlsg_frontier.cuh"

namespace vlsg {
namespace { // internal linkage: every compilation unit has its own copy

// Plane word k (-1..8) of a slot's defined mask, planes -1 and 8 from the
// z-face neighbours (0 when they are not allocated).
__device__ inline uint64_t planeOf(const uint64_t *def, int slot, int zm, int zp, int k) {
  if (k < 0) return zm >= 0 ? def[(size_t)zm * 8 + 7] : 0ull;
  if (k > 7) return zp >= 0 ? def[(size_t)zp * 8] : 0ull;
  return def[(size_t)slot * 8 + k];
}

// One Expand cycle over the defined cells that keep their value (every
// defined |value| <= the total limit): the candidates are the undefined cells
// next to a defined one.  Same results, change log, masks and visit flags as
// kFrontierPass<T, FP_EXPAND, ExpandRule<T>>.
template <class T>
__global__ void __launch_bounds__(FRONTIER_THREADS, VLSG_PASS_MIN_BLOCKS)
    kExpandRows(Topo t, LsView<T> v, ExpandRule<T> rule, ChangeLog<T> lg, const uint8_t *visitIn,
                uint8_t *visitOut) {
  __shared__ WarpScratch sm[FRONTIER_THREADS / 32]; // complex bricks only
  WarpScratch &ws = sm[threadIdx.x >> 5];
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nWarps = (gridDim.x * blockDim.x) >> 5;
  const int n = *t.nSlots;
  const size_t logBase = (size_t)warp * lg.per;
  int logged = 0;
  bool zeroHit = false;
  // rows (y, zq) and (y, zq + 4)
  const int y = lane & 7, zq = lane >> 3;
  for (int w = warp; w < n; w += nWarps) {
    const int slot = t.slotList[w];
    const bool complex = (t.cflag[slot] & CF_STAR) != 0;
    if (visitIn && !complex && !visitIn[slot]) {
      if (lane < 8) v.defNext[(size_t)slot * 8 + lane] = 0ull;
      continue;
    }
    if (complex) {
      const uint64_t own = lane < 8 ? v.def[(size_t)slot * 8 + lane] : 0ull;
      frontierBrick<T, FP_EXPAND, ExpandRule<T>>(t, v, rule, lg, ws, slot, true, own, logBase,
                                                 logged, visitOut, zeroHit);
      continue;
    }
    // face neighbours -x, +x, -y, +y, -z, +z (slot, or -1-brick)
    const int f = lane < 6 ? t.nbr[(size_t)slot * 27 + faceEntry(lane)] : 0;
    const int nxm = __shfl_sync(FULL, f, 0), nxp = __shfl_sync(FULL, f, 1);
    const int nym = __shfl_sync(FULL, f, 2), nyp = __shfl_sync(FULL, f, 3);
    const int nzm = __shfl_sync(FULL, f, 4), nzp = __shfl_sync(FULL, f, 5);
    unsigned own2 = 0, cand2 = 0; // byte h: row (y, zq + 4h)
    bool open = false;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int z = zq + 4 * h;
      const uint64_t P = v.def[(size_t)slot * 8 + z];
      const unsigned own = (unsigned)(P >> (8 * y)) & 0xffu;
      const unsigned ym = y > 0 ? (unsigned)(P >> (8 * (y - 1))) & 0xffu
                                : (nym >= 0 ? (unsigned)(v.def[(size_t)nym * 8 + z] >> 56) : 0u);
      const unsigned yp = y < 7 ? (unsigned)(P >> (8 * (y + 1))) & 0xffu
                                : (nyp >= 0 ? (unsigned)v.def[(size_t)nyp * 8 + z] & 0xffu : 0u);
      const unsigned zm = (unsigned)(planeOf(v.def, slot, nzm, nzp, z - 1) >> (8 * y)) & 0xffu;
      const unsigned zp = (unsigned)(planeOf(v.def, slot, nzm, nzp, z + 1) >> (8 * y)) & 0xffu;
      const unsigned xm =
          nxm >= 0 ? (unsigned)(v.def[(size_t)nxm * 8 + z] >> (8 * y + 7)) & 1u : 0u;
      const unsigned xp =
          nxp >= 0 ? ((unsigned)(v.def[(size_t)nxp * 8 + z] >> (8 * y)) & 1u) << 7 : 0u;
      const unsigned dil = ((own << 1) | (own >> 1) | ym | yp | zm | zp | xm | xp) & 0xffu;
      own2 |= own << (8 * h);
      cand2 |= (dil & ~own) << (8 * h);
      // a defined cell on a face whose neighbour brick is not allocated
      open |= ((own & 1u) && nxm < 0) || ((own & 0x80u) && nxp < 0) ||
              (own && ((y == 0 && nym < 0) || (y == 7 && nyp < 0) || (z == 0 && nzm < 0) ||
                       (z == 7 && nzp < 0)));
    }
    if (__any_sync(FULL, open) && lane == 0) atomicOr(t.err, 64);
    const T *bv = v.vals + (size_t)slot * BV;
    unsigned pend = cand2, born = 0;
    while (__any_sync(FULL, pend != 0u)) {
      bool changed = false;
      T out = T(0);
      uint32_t cell = 0;
      int32_t ps = -1;
      T pv = T(0), pdi = T(0);
      if (pend) {
        const int b = __ffs(pend) - 1;
        pend &= pend - 1;
        const int x = b & 7, z = zq + 4 * (b >> 3);
        const int c = z * 64 + y * 8 + x;
        const T center = bv[c];
        T nb[6]; // +x, +y, +z, -x, -y, -z
        nb[0] = x < 7 ? bv[c + 1] : refValue<T>(v.vals, v.farSign, nxp, c - 7);
        nb[1] = y < 7 ? bv[c + 8] : refValue<T>(v.vals, v.farSign, nyp, c - 56);
        nb[2] = z < 7 ? bv[c + 64] : refValue<T>(v.vals, v.farSign, nzp, c - 448);
        nb[3] = x > 0 ? bv[c - 1] : refValue<T>(v.vals, v.farSign, nxm, c + 7);
        nb[4] = y > 0 ? bv[c - 8] : refValue<T>(v.vals, v.farSign, nym, c + 56);
        nb[5] = z > 0 ? bv[c - 64] : refValue<T>(v.vals, v.farSign, nzm, c + 448);
        int src = -1;
        out = rule(center, nb, src);
        changed = out != center || signbit(out) != signbit(center);
        if (changed && isDef(out)) born |= 1u << b;
        cell = ((uint32_t)slot << 9) | (uint32_t)c;
        if (changed && lg.pd.src && isDef(out) && src >= 0) {
          // the neighbour the value came from: (slot, cell) through the faces
          const int d = src % 3, sgn = src < 3 ? 1 : -1;
          const int coord = d == 0 ? x : d == 1 ? y : z;
          const int step = d == 0 ? 1 : d == 1 ? 8 : 64;
          const bool inside = sgn > 0 ? coord < 7 : coord > 0;
          const int ref = inside ? slot
                                 : (d == 0 ? (sgn > 0 ? nxp : nxm)
                                           : d == 1 ? (sgn > 0 ? nyp : nym) : (sgn > 0 ? nzp : nzm));
          const int loc = inside ? c + sgn * step : c - sgn * 7 * step;
          payloadOf<T>(v.pd, (size_t)slot * BV + c, src, ref, loc, ps, pv, pdi);
        }
      }
      logChange<T>(lg, logBase, logged, changed, cell, out, ps, pv, pdi);
    }
    // new masks: the 8 lanes of a plane group OR their rows into the word
    const unsigned now = own2 | born;
    uint64_t W[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      uint64_t word = (uint64_t)((now >> (8 * h)) & 0xffu) << (8 * y);
      word |= __shfl_xor_sync(FULL, word, 1);
      word |= __shfl_xor_sync(FULL, word, 2);
      word |= __shfl_xor_sync(FULL, word, 4);
      W[h] = word;
      if (y == 0) v.defNext[(size_t)slot * 8 + zq + 4 * h] = word;
    }
    if (visitOut) {
      const bool rep = y == 0;
      const uint64_t both = W[0] | W[1];
      const unsigned self = __ballot_sync(FULL, rep && both != 0ull);
      const unsigned bxm = __ballot_sync(FULL, rep && (both & XLO) != 0ull);
      const unsigned bxp = __ballot_sync(FULL, rep && (both & XHI) != 0ull);
      const unsigned bym = __ballot_sync(FULL, rep && (both & 0xffull) != 0ull);
      const unsigned byp = __ballot_sync(FULL, rep && (both >> 56) != 0ull);
      const unsigned bzm = __ballot_sync(FULL, rep && zq == 0 && W[0] != 0ull);
      const unsigned bzp = __ballot_sync(FULL, rep && zq == 3 && W[1] != 0ull);
      if (lane == 0 && self) {
        visitOut[slot] = 1;
        if (bxm && nxm >= 0) visitOut[nxm] = 1;
        if (bxp && nxp >= 0) visitOut[nxp] = 1;
        if (bym && nym >= 0) visitOut[nym] = 1;
        if (byp && nyp >= 0) visitOut[nyp] = 1;
        if (bzm && nzm >= 0) visitOut[nzm] = 1;
        if (bzp && nzp >= 0) visitOut[nzp] = 1;
      }
    }
  }
  if (lane == 0) lg.count[warp] = logged;
}

} // namespace
} // namespace vlsg
