// vlsg_engine.cuh -- host orchestration of one context (templated on the
// storage type T = double or float).  Follows viennals::Advect::apply and
// the AdvectTimeIntegration schemes (lsAdvect.hpp:199-830,
// lsAdvectIntegrationSchemes.hpp:46-168) stage by stage, with every
// level-set operation running as kernels on the context stream.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstring>
#include <functional>
#include <limits>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "vlsg_common.cuh"
#include "vlsg_exchange.cuh"
#include "vlsg_iface.h"
#include "vlsg_metrics.cuh"
#include "vlsg_frontier.cuh"
#include "vlsg_maint.cuh"
#include "vlsg_passes.cuh"
#include "vlsg_rates.cuh"
#include "vlsg_batch.cuh"
#include "vlsg_velcb.cuh"
#include "vlsg_voids.cuh"

namespace vlsg {
namespace { // internal linkage: every compilation unit has its own copy

inline uint64_t hostCellKey(int x, int y, int z) {
  const uint64_t off = 1ull << 20;
  return ((uint64_t)(z + (int)off) << 42) | ((uint64_t)(y + (int)off) << 21) |
         (uint64_t)(x + (int)off);
}

template <class T> class Engine : public EngineBase {
public:
  GridDev g{};
  int L = 0;
  int nBricks = 0;
  int cap = 0; // slot capacity
  size_t poolCells = 0; // cap * 512
  // device arrays
  int *brickMap = nullptr, *slotBrick = nullptr, *slotList = nullptr;
  int *freeStack = nullptr, *newList = nullptr;
  int *counters = nullptr; // see the *Ptr() accessors
  uint8_t *needed = nullptr;
  unsigned long long *scal = nullptr;   // 0 minStep, 1..3 alphas
  unsigned long long *defCnt = nullptr; // defined cells per buffer (counted on demand)
  unsigned long long *rateCounts = nullptr; // active cells, band cells of the last rates
  int *nbr = nullptr;                   // 27 per slot
  int *slotDom = nullptr;               // batching form: the domain of each slot
  uint8_t *cflag = nullptr;             // CF_* per slot
  uint8_t *core = nullptr;              // per brick: holds an uploaded point
  unsigned long long *small = nullptr;  // 0..5 point box, 6.. |value| bounds per level set
  uint64_t *runKeys[VLSG_MAX_LEVEL_SETS] = {};
  size_t capRunKeys[VLSG_MAX_LEVEL_SETS] = {};
  // allocated sizes: arrays per brick of the map box, per slot, rate chains
  size_t capBricks = 0, capSlots = 0;
  int capL = 0;
  struct DBuf {
    T *vals = nullptr;
    uint64_t *def[2] = {nullptr, nullptr};
    int8_t *farSign = nullptr;
    size_t capSlots = 0, capBricks = 0;
    int cur = 0;
    int width = 1;
    bool live = false;
    double bound = 0;  // upper bound of |value| over the defined cells
    int64_t nDef = 0;  // defined cells (profiling mode)
    float *lo = nullptr; // compensation terms (FP32 top level set and its RK copy)
    size_t capLo = 0;
  };
  DBuf buf[MAXB];
  // rates of the active points, compact: rateCap entries per chain entry
  // (L of them), found per slot through rateBase (vlsg_rates.cuh)
  T *rateV = nullptr, *rateStop = nullptr;
  uint8_t *rateLen = nullptr;
  unsigned long long *rateBase = nullptr; // per slot
  size_t rateCap = 0;
  int rateL = 0;
  uint64_t *act = nullptr;  // active masks of the top level set
  // change log of a pass: one segment of logPer entries per warp of the pass
  uint32_t *logCell = nullptr;
  T *logVal = nullptr;
  int *logCount = nullptr;
  size_t logPer = 0;
  int logSegments = 0;
  // per buffer: the bricks its next frontier pass must visit, written by the
  // previous pass over it (visitOk false: visit every brick).  A pass writes
  // visitSpare, which then takes the buffer's place.  Flags stay valid while
  // the defined cells only shrink (they over-approximate).
  uint8_t *visit[MAXB] = {};
  uint8_t *visitSpare = nullptr;
  bool visitOk[MAXB] = {};
  void dropVisits() {
    for (bool &v : visitOk) v = false;
  }
  const uint8_t *visitIn(int b) const { return visitOk[b] ? visit[b] : nullptr; }
  uint8_t *visitOut() {
    VLSG_CUDA(cudaMemsetAsync(visitSpare, 0, cap, stream));
    return visitSpare;
  }
  void visitDone(int b) {
    std::swap(visit[b], visitSpare);
    visitOk[b] = true;
  }
  void copyVisits(int src, int dst) {
    visitOk[dst] = visitOk[src];
    if (visitOk[src])
      VLSG_CUDA(cudaMemcpyAsync(visit[dst], visit[src], cap, cudaMemcpyDeviceToDevice, stream));
  }
  // host mirrors
  int hCounters[16];
  unsigned long long hScal[4];
  int *pinCounters = nullptr;
  unsigned long long *pinScal = nullptr;
  // bookkeeping
  uint64_t launches = 0;
  int64_t lastBand = 0, lastActive = 0; // profiling: band / active cells of the stage
  uint64_t pointUpdates = 0;
  uint32_t stages = 0;
  double currentTimeStep = -1.;
  // grids of one wave: every block of a pass (and of the rate kernel) is
  // resident at once, so no tail of late blocks
  int numSMs = 148;
  int blocksPass = 148 * VLSG_PASS_MIN_BLOCKS;
  int blocksRate = 148 * rateMinBlocks<T>();
  int blocksRateWeno = 148 * rateMinBlocks<T, FAM_WENO>();
  // exchange format (points and runs in HRLE order), cached per buffer until
  // the level sets change
  struct Scratch {
    void *p = nullptr;
    size_t bytes = 0;
  };
  enum { X_FLAGS, X_POS, X_OB, X_BOUNDS, X_C, X_P, X_SUMS, X_BOX, X_IDX, X_VAL, X_GC, X_GE,
         X_ROWC, X_ROWG, X_PB, X_GB, X_RSTART, X_RSIGN, X_RPB, X_KEEP, X_KPOS, X_OSTART,
         X_OSIGN, X_VCNT, X_VOFF, X_VSUMS, X_QC, X_QM, X_QN, X_QP, X_VS, X_VV, X_AD, X_AM,
         X_AC, X_AV, X_SKEY, X_SALPHA, X_QC2, X_QN2, X_QM2, X_QP2, X_VS2, X_VPARENT, X_VMASK,
         X_VTOP, X_PSRC, X_PVEL, X_PDISS, X_SCAN2, X_COUNT };
  // pinned host staging of the velocity callback's queries and answers
  struct PinScratch {
    void *p = nullptr;
    size_t bytes = 0;
  };
  enum { H_QC, H_QM, H_QN, H_QP, H_VS, H_VV, H_AD, H_AM, H_AC, H_AV, H_COUNT };
  PinScratch hs[H_COUNT];
  Scratch xs[X_COUNT];
  uint64_t generation = 0;
  int xBuf = -1;
  uint64_t xGen = ~0ull;
  int64_t xPoints = 0, xRuns = 0;

  ~Engine() {
    release();
    for (auto &x : xs)
      if (x.p) cudaFree(x.p);
    for (auto &h : hs)
      if (h.p) cudaFreeHost(h.p);
  }

  void release() {
    dropGraphs();
    auto f = [](void *p) { if (p) cudaFree(p); };
    for (auto &b : buf) f(b.lo);
    f(brickMap); f(slotBrick); f(slotList); f(freeStack); f(newList); f(counters); f(needed);
    f(scal); f(defCnt); f(rateCounts); f(nbr); f(cflag); f(core); f(small); f(rateV);
    f(rateStop); f(rateLen); f(act); f(logCell); f(logVal); f(logCount); f(visitSpare);
    f(slotDom); slotDom = nullptr;
    f(rateBase); rateBase = nullptr; rateCap = 0; rateL = 0;
    f(domDev); f(domOfBzDev); f(domDelta); f(domVelDev); f(domRed); f(domUpdates); f(domDt);
    f(domRedInit);
    domDev = nullptr, domOfBzDev = nullptr, domDelta = nullptr, domVelDev = nullptr;
    domRed = nullptr, domUpdates = nullptr, domDt = nullptr, domRedInit = nullptr, nDom = 0;
    freePayload(pdCells);
    freePayload(pdLog);
    f(rateD);
    rateD = nullptr;
    capPdCells = capPdLog = capRateD = 0;
    for (auto &v : visit) {
      f(v);
      v = nullptr;
    }
    visitSpare = nullptr;
    dropVisits();
    for (auto &k : runKeys) f(k);
    for (auto &b : buf) {
      f(b.vals); f(b.def[0]); f(b.def[1]); f(b.farSign);
      b = DBuf();
    }
    if (pinCounters) cudaFreeHost(pinCounters);
    if (pinScal) cudaFreeHost(pinScal);
    brickMap = slotBrick = slotList = freeStack = newList = counters = nullptr;
    needed = nullptr; scal = defCnt = rateCounts = small = nullptr; nbr = nullptr;
    cflag = core = nullptr; rateV = rateStop = nullptr; rateLen = nullptr; act = nullptr;
    logCell = nullptr; logVal = nullptr; logCount = nullptr; logPer = 0; logSegments = 0;
    pinCounters = nullptr; pinScal = nullptr;
    for (int l = 0; l < VLSG_MAX_LEVEL_SETS; ++l) runKeys[l] = nullptr, capRunKeys[l] = 0;
    capBricks = capSlots = 0;
    capL = 0;
  }

  int *nSlotsPtr() { return counters + 0; }
  int *freeCountPtr() { return counters + 1; }
  int *nActivePtr() { return counters + 2; }
  int *errPtr() { return counters + 3; }
  int *flagPtr() { return counters + 4; }
  int *nOutPtr() { return counters + 5; }
  int *nNewPtr() { return counters + 10; }
  int *zeroPtr() { return counters + 14; } // a Prune pass met a defined +-0

  MapView mapView() const { return MapView{brickMap, slotBrick}; }
  Buf<T> view(int b) const { return Buf<T>{buf[b].vals, buf[b].farSign}; }
  Topo topo() { return Topo{g, brickMap, slotBrick, slotList, nSlotsPtr(), nbr, cflag, errPtr()}; }
  LsView<T> lsView(int b) {
    auto &B = buf[b];
    return LsView<T>{B.vals, B.def[B.cur], B.def[1 - B.cur], B.farSign, payloadOf(b)};
  }
  ChangeLog<T> changeLog(int b) {
    return ChangeLog<T>{logCell, logVal, logCount, logPer,
                        pdTracked(b) ? pdLog : Payload<T>{nullptr, nullptr, nullptr}};
  }

  // --------------------------------------------------------- point data
  // The top level set's point data through an advection: per cell of its
  // buffer the source id and the saved velocity / dissipation, carried by
  // every pass through its change log (pdLog), set at the start of
  // vlsg_advect from the points' ranks and by the value update.
  Payload<T> pdCells{}, pdLog{};
  size_t capPdCells = 0, capPdLog = 0;
  T *rateD = nullptr;
  size_t capRateD = 0;
  bool pdTrack = false; // carried through this advection
  bool pdSave = false;  // saved velocities (setSaveAdvectionVelocities)
  bool pdHas = false;   // the top level set carries point data now
  bool pdTracked(int b) const { return pdTrack && b == L - 1; }
  Payload<T> payloadOf(int b) const {
    return pdTracked(b) ? pdCells : Payload<T>{nullptr, nullptr, nullptr};
  }
  static void freePayload(Payload<T> &p) {
    if (p.src) cudaFree(p.src);
    if (p.vel) cudaFree(p.vel);
    if (p.diss) cudaFree(p.diss);
    p = Payload<T>{nullptr, nullptr, nullptr};
  }
  static void allocPayload(Payload<T> &p, size_t &cap, size_t n) {
    if (cap >= n && p.src) return;
    freePayload(p);
    VLSG_CUDA(cudaMalloc(&p.src, n * sizeof(int32_t)));
    VLSG_CUDA(cudaMalloc(&p.vel, n * sizeof(T)));
    VLSG_CUDA(cudaMalloc(&p.diss, n * sizeof(T)));
    cap = n;
  }
  // Start of an advection with point data: every defined cell of the top
  // level set carries its own rank (the order of vlsg_download_levelset).
  void initPointData() {
    const int top = L - 1;
    allocPayload(pdCells, capPdCells, poolCells);
    allocPayload(pdLog, capPdLog, logPer * (size_t)logSegments);
    if (pdSave) growDevice(rateD, capRateD, std::max<size_t>(rateCap, 1) * (size_t)L);
    const int nList = readI32(nSlotsPtr());
    xBuf = -1; // the point layout below reuses the exchange's scratch
    pointLayout(top, nList);
    const PointRanks R{slotBrick, (const uint32_t *)xs[X_POS].p, (const int4 *)xs[X_BOUNDS].p,
                       (const uint32_t *)xs[X_P].p, buf[top].def[buf[top].cur]};
    Scope sc(this, "point_data");
    kInitPointData<T><<<blocksPass, 256, 0, stream>>>(slotList, nSlotsPtr(),
                                                      buf[top].def[buf[top].cur], R, pdCells);
    checkLaunch();
  }

  // ---------------------------------------------------------------- timing
  // One kernel launch.  With profiling on it is bracketed by CUDA events on
  // the context stream and, after the kernel finished, `bytesFn` turns the
  // device counters into the launch's algorithmic bytes.
  struct Scope {
    Engine *e;
    int idx;
    cudaEvent_t a, b;
    std::function<double()> bytesFn;
    Scope(Engine *eng, const char *name, std::function<double()> fn = nullptr)
        : e(eng), idx(-1), bytesFn(std::move(fn)) {
      ++e->launches;
      if (!e->profiling) return;
      for (size_t i = 0; i < e->timers.size(); ++i)
        if (e->timers[i].name == name) idx = (int)i;
      if (idx < 0) {
        e->timers.push_back(KernelTimer{name});
        idx = (int)e->timers.size() - 1;
      }
      e->timers[idx].launches++;
      cudaEventCreate(&a);
      cudaEventCreate(&b);
      cudaEventRecord(a, e->stream);
    }
    ~Scope() {
      if (!e->profiling || idx < 0) return;
      cudaEventRecord(b, e->stream);
      cudaEventSynchronize(b);
      float ms = 0;
      cudaEventElapsedTime(&ms, a, b);
      e->timers[idx].ms += ms;
      cudaEventDestroy(a);
      cudaEventDestroy(b);
      if (bytesFn) e->timers[idx].bytes += bytesFn();
    }
  };
  // Stream-ordered reads of device counters (synchronous).
  unsigned long long readU64(const unsigned long long *p) {
    VLSG_CUDA(cudaMemcpyAsync(pinScal + 7, p, sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream));
    VLSG_CUDA(cudaStreamSynchronize(stream));
    return pinScal[7];
  }
  int readI32(const int *p) {
    VLSG_CUDA(cudaMemcpyAsync(pinCounters + 31, p, sizeof(int), cudaMemcpyDeviceToHost, stream));
    VLSG_CUDA(cudaStreamSynchronize(stream));
    return pinCounters[31];
  }
  // Defined cells of buffer b, counted from its masks (synchronous; for the
  // download and the profiling byte counts).
  int64_t defined(int b) {
    VLSG_CUDA(cudaMemsetAsync(defCnt + b, 0, sizeof(unsigned long long), stream));
    kCountDefined<<<grid1(cap), 256, 0, stream>>>(slotList, nSlotsPtr(), buf[b].def[buf[b].cur],
                                                  defCnt + b);
    checkLaunch();
    return (int64_t)readU64(defCnt + b);
  }
  // Bytes of a band pass in the survey's accounting: value + 64-bit key,
  // read once and written once per band point.
  double bandPassBytes(int64_t nIn, int64_t nOut) const {
    return double(sizeof(T) + 8) * double(nIn + nOut);
  }
  void checkLaunch() { VLSG_CUDA(cudaGetLastError()); }

  static int grid1(size_t n) {
    size_t b = (n + 255) / 256;
    if (b < 1) b = 1;
    if (b > 148 * 32) b = 148 * 32;
    return (int)b;
  }

  // ------------------------------------------------------------- layout
  // Arrays of buffers 0..nb-1 at the current sizes (contents of a grown
  // array are not kept; every build fills them).
  void allocBuffers(int nb) {
    for (int b = 0; b < nb; ++b) {
      auto &B = buf[b];
      if (B.capSlots < capSlots || !B.vals) {
        if (B.vals) VLSG_CUDA(cudaFree(B.vals));
        if (B.def[0]) VLSG_CUDA(cudaFree(B.def[0]));
        if (B.def[1]) VLSG_CUDA(cudaFree(B.def[1]));
        B.vals = nullptr, B.def[0] = B.def[1] = nullptr;
        VLSG_CUDA(cudaMalloc(&B.vals, capSlots * BV * sizeof(T)));
        VLSG_CUDA(cudaMalloc(&B.def[0], capSlots * 8 * sizeof(uint64_t)));
        VLSG_CUDA(cudaMalloc(&B.def[1], capSlots * 8 * sizeof(uint64_t)));
        B.capSlots = capSlots;
      }
      if (B.capBricks < capBricks || !B.farSign) {
        if (B.farSign) VLSG_CUDA(cudaFree(B.farSign));
        B.farSign = nullptr;
        VLSG_CUDA(cudaMalloc(&B.farSign, capBricks));
        B.capBricks = capBricks;
      }
      if (loWanted && hasLo(b) && (B.capLo < capSlots || !B.lo)) {
        if (B.lo) VLSG_CUDA(cudaFree(B.lo));
        B.lo = nullptr;
        VLSG_CUDA(cudaMalloc(&B.lo, capSlots * BV * sizeof(float)));
        B.capLo = capSlots;
      }
    }
  }
  // The precision form (T = float) can keep, for the top level set and its RK
  // copy, a second FP32 array per cell: the compensation term `lo` of the
  // value, whose exact value is hi + lo.  Only the value update and the RK
  // stage combination (both in double) produce a non-zero term; every other
  // write of a value (a pass's change, a boolean, a copy without terms) sets
  // it to zero, so that hi + lo is always the value the FP64 arithmetic of
  // those two steps produced or the stored value itself.  Stencils and pass
  // rules read hi only; downloads and queries return hi + lo.
  // The terms are kept only by operations run with compensation on (an
  // upload, an advection with fp32_compensation); loValid tells whether the
  // arrays are current for downloads and queries.  An advection with
  // compensation that finds them stale starts from zero terms (value = hi).
  static constexpr bool kComp = sizeof(T) == 4;
  bool compActive = false;
  bool loValid = false;
  bool loWanted = false; // the arrays exist only once compensation was asked for
  // the uploaded top level set (device arrays of the context) while the
  // level sets are unchanged since the upload: its doubles give the first
  // compensation terms
  const int32_t *upIdx = nullptr;
  const double *upVals = nullptr;
  int64_t upN = 0;
  bool pristine = false;
  bool hasLo(int b) const { return kComp && (b == L - 1 || b == 2 * L - 1); }
  float *loOf(int b) { return compActive && hasLo(b) ? buf[b].lo : nullptr; }
  const float *loRead(int b) const { return loValid && hasLo(b) ? buf[b].lo : nullptr; }

  // The live buffers (current level sets and the RK copies in use).
  BufSet bufSet() {
    BufSet s{};
    int k = 0;
    for (int b = 0; b < 2 * L; ++b) {
      if (!buf[b].live || !buf[b].vals) continue;
      s.vals[k] = buf[b].vals;
      s.def[k] = buf[b].def[buf[b].cur];
      s.farSign[k] = buf[b].farSign;
      ++k;
    }
    s.nBuf = k;
    return s;
  }

  // Per-brick arrays for nb bricks and per-slot arrays for c slots; cap
  // becomes the allocated slot count.
  void ensureLayout(size_t nb, size_t c) {
    if (nb > capBricks) {
      for (void *p : {(void *)brickMap, (void *)needed, (void *)core})
        if (p) VLSG_CUDA(cudaFree(p));
      brickMap = nullptr, needed = nullptr, core = nullptr;
      const size_t n = nb + nb / 4 + 64;
      VLSG_CUDA(cudaMalloc(&brickMap, n * sizeof(int)));
      VLSG_CUDA(cudaMalloc(&needed, n));
      VLSG_CUDA(cudaMalloc(&core, n));
      capBricks = n;
    }
    if (c > 0 && (c > capSlots || L > capL)) {
      for (void *p : {(void *)slotBrick, (void *)slotList, (void *)freeStack, (void *)newList,
                      (void *)nbr, (void *)cflag, (void *)act, (void *)logCell, (void *)logVal,
                      (void *)logCount, (void *)visitSpare, (void *)slotDom, (void *)rateBase})
        if (p) VLSG_CUDA(cudaFree(p));
      for (auto &v : visit) {
        if (v) VLSG_CUDA(cudaFree(v));
        v = nullptr;
      }
      slotBrick = slotList = freeStack = newList = nbr = logCount = nullptr;
      cflag = nullptr, act = nullptr, logCell = nullptr, slotDom = nullptr, rateBase = nullptr;
      logVal = nullptr;
      const size_t n = std::max(c, capSlots);
      const int l = std::max(L, capL);
      VLSG_CUDA(cudaMalloc(&slotBrick, n * sizeof(int)));
      VLSG_CUDA(cudaMalloc(&slotList, n * sizeof(int)));
      VLSG_CUDA(cudaMalloc(&freeStack, n * sizeof(int)));
      VLSG_CUDA(cudaMalloc(&newList, n * sizeof(int)));
      VLSG_CUDA(cudaMalloc(&nbr, n * 27 * sizeof(int)));
      VLSG_CUDA(cudaMalloc(&cflag, n));
      VLSG_CUDA(cudaMalloc(&slotDom, n * sizeof(int)));
      VLSG_CUDA(cudaMalloc(&act, n * 8 * sizeof(uint64_t)));
      // pass grids: one wave of the GPU, or one warp per 8 slots for small
      // pools (the change log holds a segment per warp)
      blocksPass = std::min(numSMs * VLSG_PASS_MIN_BLOCKS,
                            std::max(numSMs, (int)((n + 63) / 64)));
      // a pass warp handles at most ceil(n / warps) bricks: its log segment
      // holds all their cells
      logSegments = blocksPass * (FRONTIER_THREADS / 32);
      logPer = (size_t)BV * ((n + logSegments - 1) / logSegments);
      VLSG_CUDA(cudaMalloc(&logCell, logPer * logSegments * sizeof(uint32_t)));
      VLSG_CUDA(cudaMalloc(&logVal, logPer * logSegments * sizeof(T)));
      VLSG_CUDA(cudaMalloc(&logCount, logSegments * sizeof(int)));
      for (auto &v : visit) VLSG_CUDA(cudaMalloc(&v, n));
      VLSG_CUDA(cudaMalloc(&visitSpare, n));
      dropVisits();
      VLSG_CUDA(cudaMalloc(&rateBase, n * sizeof(unsigned long long)));
      capSlots = n;
      capL = l;
    }
    cap = (int)capSlots;
    poolCells = (size_t)cap * BV;
  }

  // Compact rate arrays for at least n active points and L chain entries
  // (the saved dissipation too with setSaveAdvectionVelocities).
  void ensureRateCap(size_t n) {
    if (n <= rateCap && L <= rateL && rateV && (!pdSave || (rateD && capRateD >= rateCap * L)))
      return;
    const size_t c = std::max(n, rateCap);
    const int l = std::max(L, rateL);
    for (void *p : {(void *)rateV, (void *)rateStop, (void *)rateLen})
      if (p) VLSG_CUDA(cudaFree(p));
    rateV = rateStop = nullptr, rateLen = nullptr;
    VLSG_CUDA(cudaMalloc(&rateV, c * l * sizeof(T)));
    VLSG_CUDA(cudaMalloc(&rateStop, c * l * sizeof(T)));
    VLSG_CUDA(cudaMalloc(&rateLen, c));
    rateCap = c, rateL = l;
    if (pdSave) growDevice(rateD, capRateD, c * l);
    dropGraphs(); // captured steps hold the old arrays
  }

  void ensureSmall() {
    if (counters) return;
    int dev = 0;
    VLSG_CUDA(cudaGetDevice(&dev));
    VLSG_CUDA(cudaDeviceGetAttribute(&numSMs, cudaDevAttrMultiProcessorCount, dev));
    blocksPass = numSMs * VLSG_PASS_MIN_BLOCKS;
    blocksRate = numSMs * rateMinBlocks<T>();
    blocksRateWeno = numSMs * rateMinBlocks<T, FAM_WENO>();
    VLSG_CUDA(cudaHostAlloc(&pinCounters, 32 * sizeof(int), cudaHostAllocDefault));
    VLSG_CUDA(cudaHostAlloc(&pinScal, 32 * sizeof(unsigned long long), cudaHostAllocDefault));
    VLSG_CUDA(cudaMalloc(&counters, 16 * sizeof(int)));
    VLSG_CUDA(cudaMalloc(&scal, 4 * sizeof(unsigned long long)));
    VLSG_CUDA(cudaMalloc(&defCnt, MAXB * sizeof(unsigned long long)));
    VLSG_CUDA(cudaMalloc(&rateCounts, 4 * sizeof(unsigned long long))); // active, band, rate entries
    VLSG_CUDA(cudaMalloc(&small, 16 * sizeof(unsigned long long)));
  }

  // Lay the uploaded level sets out on the device (lsDomain's HRLE data
  // becomes bricks): map box from the points, allocated bricks = the
  // points' bricks and their neighbours, values from the points and the
  // runs' signs.  Allocations are reused from the previous build when they
  // are large enough.
  void build(const GridDev &grid, std::vector<StagedLS> &ls, int margin) override {
    ++generation;
    dropGraphs(); // captured steps hold the old layout's pointers
    batchSteps = 0;
    dropVisits();
    pdTrack = pdSave = pdHas = false;
    ensureSmall();
    g = grid;
    L = (int)ls.size();
    VLSG_CUDA(cudaMemsetAsync(counters, 0, 16 * sizeof(int), stream));
    // point box (through the boundary mapping), run keys, order check
    const int boxInit[6] = {INT_MAX, INT_MAX, INT_MAX, INT_MIN, INT_MIN, INT_MIN};
    std::memcpy(pinCounters + 16, boxInit, sizeof(boxInit));
    int *box = (int *)small;
    VLSG_CUDA(cudaMemcpyAsync(box, pinCounters + 16, sizeof(boxInit), cudaMemcpyHostToDevice, stream));
    for (int l = 0; l < L; ++l) {
      auto &s = ls[l];
      if (s.n) {
        Scope sc(this, "upload_points");
        kStagePoints<<<grid1(s.n), 256, 0, stream>>>(g, (int)s.n, s.idx, box, errPtr());
        checkLaunch();
      }
      growDevice(runKeys[l], capRunKeys[l], (size_t)s.nRuns);
      if (s.nRuns) {
        Scope sc(this, "upload_runs");
        kStageRuns<<<grid1(s.nRuns), 256, 0, stream>>>((int)s.nRuns, s.runStart, runKeys[l],
                                                       counters + 12 /* unsorted flag */);
        checkLaunch();
      }
    }
    VLSG_CUDA(cudaMemcpyAsync(pinCounters + 16, box, sizeof(boxInit), cudaMemcpyDeviceToHost, stream));
    syncErr("upload");
    int hb[6];
    std::memcpy(hb, pinCounters + 16, sizeof(hb));
    if (hCounters[12]) sortRuns(ls);
    // box: bounded directions cover the grid, infinite ones the points + margin
    // (the batching form brings its box with the domain table)
    for (int d = 0; d < 3 && !g.nDom; ++d) {
      const bool bounded = g.bc[d] == VLSG_PERIODIC_BOUNDARY || g.bc[d] == VLSG_REFLECTIVE_BOUNDARY;
      if (bounded) {
        g.org[d] = g.gmin[d];
        const int n = g.bc[d] == VLSG_PERIODIC_BOUNDARY ? g.gmax[d] - g.gmin[d]
                                                       : g.gmax[d] - g.gmin[d] + 1;
        g.nb[d] = (n + BS - 1) / BS;
      } else {
        long long lo = hb[d], hi = hb[3 + d];
        if (lo > hi) lo = hi = 0;
        const long long a = lo - (long long)margin * BS;
        const long long b = hi + (long long)margin * BS;
        const long long a8 = (a >= 0) ? (a / BS) * BS : -(((-a) + BS - 1) / BS) * BS;
        g.org[d] = (int)a8;
        g.nb[d] = (int)((b - a8) / BS + 1);
      }
    }
    const long long nb64 = (long long)g.nb[0] * g.nb[1] * g.nb[2];
    if (nb64 > INT_MAX / 2) throw CudaError("upload: brick box too large", VLSG_ERR_CAPACITY);
    nBricks = (int)nb64;
    ensureLayout(nBricks, 0);
    VLSG_CUDA(cudaMemsetAsync(brickMap, 0xff, nBricks * sizeof(int), stream));
    VLSG_CUDA(cudaMemsetAsync(needed, 0, nBricks, stream));
    VLSG_CUDA(cudaMemsetAsync(core, 0, nBricks, stream));
    for (int l = 0; l < L; ++l) {
      if (!ls[l].n) continue;
      Scope sc(this, "upload_mark");
      kMarkPointBricks<<<grid1(ls[l].n), 256, 0, stream>>>(g, (int)ls[l].n, ls[l].idx, core, errPtr());
      checkLaunch();
    }
    {
      Scope sc(this, "upload_dilate");
      kDilateBricks<<<grid1(nBricks), 256, 0, stream>>>(g, nBricks, core, needed, errPtr());
      kCountFlags<<<grid1(nBricks), 256, 0, stream>>>(needed, nBricks, counters + 13);
      checkLaunch();
    }
    syncErr("upload");
    const long long nNeeded = hCounters[13];
    // the pool keeps room for the band to grow: reallocate only when the
    // allocated slots fall below 1.25x the needed ones, then to 2x
    // (2x, or less where 2x would take more than about half of the free
    // device memory: every level set and its RK copy hold values and masks
    // for every slot, and the change log a share of 512 cells per slot)
    {
      const size_t minSlots = (size_t)std::max<long long>(1024, nNeeded + nNeeded / 4 + 256);
      size_t want = (size_t)std::max<long long>(1024, nNeeded * 2 + 256);
      size_t freeB = 0, totalB = 0;
      if (cudaMemGetInfo(&freeB, &totalB) == cudaSuccess) {
        const size_t perSlot = (size_t)(2 * L) * (BV * sizeof(T) + 2 * 8 * sizeof(uint64_t) + 1) +
                               (size_t)BV * (sizeof(uint32_t) + sizeof(T)) + 27 * sizeof(int) + 128;
        const size_t budget = freeB / 100 * 55 / perSlot;
        if (want > budget) want = std::max(minSlots, budget);
      }
      ensureLayout(nBricks, capSlots >= minSlots ? capSlots : want);
    }
    {
      Scope sc(this, "upload_pool");
      kInitFreeStack<<<grid1(cap), 256, 0, stream>>>(freeStack, cap);
      VLSG_CUDA(cudaMemsetAsync(slotBrick, 0xff, (size_t)cap * sizeof(int), stream));
      checkLaunch();
    }
    const int c2[2] = {0, cap};
    std::memcpy(pinCounters + 24, c2, sizeof(c2));
    VLSG_CUDA(cudaMemcpyAsync(counters, pinCounters + 24, sizeof(c2), cudaMemcpyHostToDevice, stream));
    for (auto &B : buf) {
      B.cur = 0, B.width = 1, B.live = false, B.bound = 0, B.nDef = 0;
    }
    allocBuffers(L);
    for (int l = 0; l < L; ++l) {
      Scope sc(this, "upload_farsign");
      kFarSignRows<<<grid1((size_t)g.nb[1] * g.nb[2]), 256, 0, stream>>>(g, runKeys[l], ls[l].runSign,
                                                           (int)ls[l].nRuns, buf[l].farSign);
      checkLaunch();
      buf[l].width = ls[l].width;
      buf[l].live = true;
    }
    {
      Scope sc(this, "alloc");
      kAllocNeeded<<<grid1(nBricks), 256, 0, stream>>>(nBricks, brickMap, slotBrick, needed,
                                                       freeStack, freeCountPtr(), nullptr,
                                                       nNewPtr(), errPtr());
      checkLaunch();
    }
    rebuildSlotList();
    VLSG_CUDA(cudaMemsetAsync(small + 6, 0, VLSG_MAX_LEVEL_SETS * sizeof(unsigned long long), stream));
    for (int l = 0; l < L; ++l) {
      auto &s = ls[l];
      {
        Scope sc(this, "upload_fill");
        kFillRows<T><<<grid1((size_t)cap * 64), 256, 0, stream>>>(
            g, slotList, nSlotsPtr(), slotBrick, cflag, runKeys[l], s.runSign, (int)s.nRuns,
            buf[l].vals);
        checkLaunch();
      }
      if (s.n) {
        Scope sc(this, "upload_scatter");
        kScatterPoints<T><<<grid1(s.n), 256, 0, stream>>>(g, (int)s.n, s.idx, s.vals, brickMap,
                                                          buf[l].vals, errPtr(), nullptr);
        checkLaunch();
      }
      {
        Scope sc(this, "upload_masks");
        kMasksFromValues<T><<<blocksPass, FRONTIER_THREADS, 0, stream>>>(
            g, slotBrick, slotList, nSlotsPtr(), buf[l].vals, buf[l].def[buf[l].cur], nullptr,
            small + 6 + l);
        checkLaunch();
      }
    }
    loValid = false;
    upIdx = ls[L - 1].idx, upVals = ls[L - 1].vals, upN = ls[L - 1].n;
    pristine = true;
    VLSG_CUDA(cudaMemcpyAsync(pinScal + 8, small + 6, VLSG_MAX_LEVEL_SETS * sizeof(unsigned long long),
                              cudaMemcpyDeviceToHost, stream));
    syncErr("upload");
    for (int l = 0; l < L; ++l) {
      double bound;
      std::memcpy(&bound, &pinScal[8 + l], sizeof(double));
      buf[l].bound = bound;
      buf[l].nDef = profiling ? defined(l) : 0;
    }
  }

  // Runs that arrived out of HRLE order: sort them (stable) on the host.
  void sortRuns(std::vector<StagedLS> &ls) {
    for (int l = 0; l < L; ++l) {
      auto &s = ls[l];
      if (s.nRuns < 2) continue;
      std::vector<uint64_t> k(s.nRuns);
      std::vector<int8_t> sg(s.nRuns);
      std::vector<int32_t> st(3 * s.nRuns);
      VLSG_CUDA(cudaMemcpyAsync(k.data(), runKeys[l], s.nRuns * sizeof(uint64_t), cudaMemcpyDeviceToHost, stream));
      VLSG_CUDA(cudaMemcpyAsync(sg.data(), s.runSign, s.nRuns, cudaMemcpyDeviceToHost, stream));
      VLSG_CUDA(cudaMemcpyAsync(st.data(), s.runStart, 3 * s.nRuns * sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
      VLSG_CUDA(cudaStreamSynchronize(stream));
      std::vector<int64_t> o(s.nRuns);
      for (int64_t i = 0; i < s.nRuns; ++i) o[i] = i;
      std::stable_sort(o.begin(), o.end(), [&](int64_t a, int64_t b) { return k[a] < k[b]; });
      std::vector<uint64_t> k2(s.nRuns);
      std::vector<int8_t> sg2(s.nRuns);
      std::vector<int32_t> st2(3 * s.nRuns);
      for (int64_t i = 0; i < s.nRuns; ++i) {
        k2[i] = k[o[i]], sg2[i] = sg[o[i]];
        for (int d = 0; d < 3; ++d) st2[3 * i + d] = st[3 * o[i] + d];
      }
      VLSG_CUDA(cudaMemcpyAsync(runKeys[l], k2.data(), s.nRuns * sizeof(uint64_t), cudaMemcpyHostToDevice, stream));
      VLSG_CUDA(cudaMemcpyAsync(s.runSign, sg2.data(), s.nRuns, cudaMemcpyHostToDevice, stream));
      VLSG_CUDA(cudaMemcpyAsync(s.runStart, st2.data(), 3 * s.nRuns * sizeof(int32_t), cudaMemcpyHostToDevice, stream));
      VLSG_CUDA(cudaStreamSynchronize(stream));
    }
  }

  void syncErr(const char *where) {
    VLSG_CUDA(cudaMemcpyAsync(pinCounters, counters, 16 * sizeof(int), cudaMemcpyDeviceToHost, stream));
    VLSG_CUDA(cudaStreamSynchronize(stream));
    std::memcpy(hCounters, pinCounters, sizeof(hCounters));
    const int e = hCounters[3];
    if (e) {
      std::string m = std::string(where) + ": device check failed:";
      if (e & 1) m += " band reached the edge of the brick box (infinite direction);";
      if (e & 2) m += " stop chain overran;";
      if (e & 4) m += " brick pool capacity exceeded;";
      if (e & 8) m += " freed brick held a defined point;";
      if (e & 64) m += " band reached an unallocated brick;";
      if (e & 128) m += " a point index lies outside the supported range (+-2^19);";
      if (e & 256) m += " the void search did not settle within its bound;";
      if (e & 512) m += " batching form: a domain's first stage found no positive time step;";
      if (e & 1024) m += " the rate storage was too small for the active points;";
      int z = 0;
      cudaMemcpy(errPtr(), &z, sizeof(int), cudaMemcpyHostToDevice);
      throw CudaError(m, (e & 4) ? VLSG_ERR_CAPACITY : VLSG_ERR_DEVICE_CHECK);
    }
  }

  void rebuildSlotList() {
    VLSG_CUDA(cudaMemsetAsync(nSlotsPtr(), 0, sizeof(int), stream));
    {
      Scope sc(this, "slot_list");
      kBuildSlotList<<<grid1(nBricks), 256, 0, stream>>>(nBricks, brickMap, slotList, nSlotsPtr());
      checkLaunch();
    }
    {
      Scope sc(this, "neighbours");
      kBuildNeighbours<<<grid1(cap), 256, 0, stream>>>(g, brickMap, slotBrick, slotList,
                                                       nSlotsPtr(), nbr, cflag, slotDom);
      checkLaunch();
    }
  }

  // Bring the allocated bricks back to dilate(core) of the live buffers.
  void maintain() {
    // the visit flags stay valid: freed slots leave the list, new ones are
    // marked (kVisitNewSlots), the defined masks do not change
    VLSG_CUDA(cudaMemsetAsync(needed, 0, nBricks, stream));
    {
      Scope sc(this, "maint_mark");
      kMarkNeeded<<<grid1(cap), 256, 0, stream>>>(g, slotBrick, slotList, nSlotsPtr(),
                                                  bufSet(), needed, errPtr());
      checkLaunch();
    }
    {
      Scope sc(this, "maint_free");
      kFreeUnneeded<T><<<grid1(cap), 256, 0, stream>>>(g, slotList, nSlotsPtr(), brickMap,
                                                       slotBrick, needed, bufSet(), freeStack,
                                                       freeCountPtr(), errPtr());
      checkLaunch();
    }
    VLSG_CUDA(cudaMemsetAsync(nNewPtr(), 0, sizeof(int), stream));
    {
      Scope sc(this, "maint_alloc");
      kAllocNeeded<<<grid1(nBricks), 256, 0, stream>>>(nBricks, brickMap, slotBrick, needed,
                                                       freeStack, freeCountPtr(), newList,
                                                       nNewPtr(), errPtr());
      checkLaunch();
    }
    {
      Scope sc(this, "maint_init");
      kInitNewSlots<T><<<blocksPass, 128, 0, stream>>>(g, newList, nNewPtr(), slotBrick, bufSet());
      checkLaunch();
      VisitSet vs{};
      for (int b = 0; b < MAXB; ++b)
        if (visitOk[b]) vs.p[vs.n++] = visit[b];
      if (vs.n) {
        kVisitNewSlots<<<blocksPass, 256, 0, stream>>>(newList, nNewPtr(), vs);
        checkLaunch();
      }
    }
    rebuildSlotList();
  }

  // --------------------------------------------------------------- passes
  void applyChanges(int b) {
    Scope sc(this, "apply_changes");
    kApplyChanges<T><<<logSegments, FRONTIER_THREADS, 0, stream>>>(buf[b].vals, changeLog(b),
                                                                    logSegments, loOf(b),
                                                                    payloadOf(b));
    checkLaunch();
  }

  // One star pass of `rule` over buffer b: candidates, changes, write-back.
  template <int MODE, class Rule>
  void frontierPass(int b, Rule rule, const char *name, int zeroMode = 0) {
    const int64_t nIn = profiling ? defined(b) : 0;
    {
      Scope sc(this, name, [this, b, nIn] {
        // the output band is known once the new masks are current
        buf[b].cur ^= 1;
        buf[b].nDef = defined(b);
        buf[b].cur ^= 1;
        return bandPassBytes(nIn, buf[b].nDef);
      });
      kFrontierPass<T, MODE, Rule><<<blocksPass, FRONTIER_THREADS, 0, stream>>>(
          topo(), lsView(b), rule, changeLog(b), visitIn(b), visitOut(), zeroPtr(), zeroMode, cap);
      visitDone(b);
      checkLaunch();
    }
    applyChanges(b);
    buf[b].cur ^= 1;
  }

  // Expand::apply (lsExpand.hpp:44-172)
  void expand(int b, int width) {
    if (width <= buf[b].width) return;
    const int startWidth = buf[b].width;
    const T totalLimit = T(width * 0.5);
    const int cycles = width - startWidth;
    // defined cells with |value| <= totalLimit keep their value
    const bool onlyUndefined = buf[b].bound <= (double)totalLimit;
    for (int c = 0; c < cycles; ++c) {
      ExpandRule<T> r{totalLimit, T((startWidth + c + 1) * T(0.5))};
      if (g.planar) {
        if (onlyUndefined) frontierPass<FP_EXPAND>(b, PlanarExpandRule<T>{r}, "expand");
        else frontierPass<FP_ALL>(b, PlanarExpandRule<T>{r}, "expand");
      } else if (onlyUndefined) {
        frontierPass<FP_EXPAND>(b, r, "expand");
      } else {
        frontierPass<FP_ALL>(b, r, "expand");
      }
      if (b == L - 1 && startWidth + c + 1 == saveTopAt) {
        // the RK copy of the top level set, taken at this width (saveTop)
        saveTopAt = 0;
        copyBuffer(b, 2 * L - 1);
        buf[2 * L - 1].width = startWidth + c + 1;
        buf[2 * L - 1].bound = 0.5 * (startWidth + c + 1);
      }
    }
    buf[b].width = width;
    buf[b].bound = (double)totalLimit;
  }
  // Prune with stray-zero removal, then without (lsBooleanOperation.hpp:
  // 203-210).  When the first pass meets no defined value +-0 it only turns
  // cells undefined with their sign class, and every cell it keeps keeps a
  // star neighbour of the other sign class (that neighbour is kept as well,
  // or is undefined and keeps its class): the second pass then changes
  // nothing, and its kernel only carries the masks and visit flags over.
  void prunePair(int b) {
    VLSG_CUDA(cudaMemsetAsync(zeroPtr(), 0, sizeof(int), stream));
    frontierPass<FP_PRUNE>(b, PruneRule<T>{true}, "prune", 1);
    frontierPass<FP_PRUNE>(b, PruneRule<T>{false}, "prune", 2);
    buf[b].width = 2;
  }
  void prune(int b, bool rsz) {
    frontierPass<FP_PRUNE>(b, PruneRule<T>{rsz}, "prune");
    buf[b].width = 2;
  }
  // rebuildLS: cutoff 1 and width 2, or 1.5 and 3 for StencilLocalLaxFriedrichs
  // (lsAdvect.hpp:250-256)
  double rebuildCutoff = 1.0;
  int rebuildWidth = 2;
  void rebuild(int b) {
    frontierPass<FP_ALL>(b, RebuildRule<T>{T(rebuildCutoff)}, "rebuild");
    buf[b].width = rebuildWidth;
    buf[b].bound = 1.0;
  }
  // updateLevelSet (value update + Reduce(1)) followed by rebuildLS
  // domDts (batching form): the time step per domain instead of dt
  void updateRebuild(double dt, const double *domDts = nullptr) {
    const int top = L - 1;
    {
      // active values read and written, their rates read
      Scope sc(this, "update", [this] { return 3.0 * double(sizeof(T)) * double(lastActive); });
      kUpdate<T><<<blocksPass, RATE_THREADS, 0, stream>>>(slotList, nSlotsPtr(), act, buf[top].vals,
                                                          rateV, rateStop, rateLen, rateBase, rateCap, L,
                                                          dt, errPtr(), loOf(top),
                                                          pdSave ? pdCells.vel : nullptr,
                                                          pdSave ? pdCells.diss : nullptr,
                                                          pdSave ? rateD : nullptr,
                                                          domDts ? slotDom : nullptr, domDts);
      checkLaunch();
    }
    {
      Scope sc(this, "update_rebuild", [this, top] {
        buf[top].cur ^= 1;
        buf[top].nDef = defined(top);
        buf[top].cur ^= 1;
        // in: the active band; out: the new band
        return bandPassBytes(lastActive, buf[top].nDef);
      });
      kUpdateRebuild<T><<<blocksPass, FRONTIER_THREADS, 0, stream>>>(
          topo(), lsView(top), act, rebuildCutoff, changeLog(top), visitIn(top), visitOut());
      visitDone(top);
      checkLaunch();
    }
    applyChanges(top);
    buf[top].cur ^= 1;
    buf[top].width = rebuildWidth;
    buf[top].bound = 1.0;
    ++stages;
  }
  template <class Comp> void pointwise(int a, int bb, Comp comp, int *flag) {
    // a combination that only undefines cells keeps a's flags valid
    if (!Comp::keepsUndefinedA) visitOk[a] = false;
    {
      const int64_t nA = profiling ? defined(a) : 0, nB = profiling ? defined(bb) : 0;
      Scope sc(this, "boolean", [this, a, nA, nB] {
        buf[a].nDef = defined(a);
        return bandPassBytes(nA + nB, buf[a].nDef);
      });
      if constexpr (Comp::keepsUndefinedA) {
        kPointwiseDefined<T, Comp><<<blocksPass, FRONTIER_THREADS, 0, stream>>>(
            topo(), buf[a].vals, buf[a].def[buf[a].cur], buf[bb].vals, comp, flag, loOf(a),
            loOf(bb));
      } else {
        kPointwise<T, Comp><<<blocksPass, FRONTIER_THREADS, 0, stream>>>(
            topo(), buf[a].vals, buf[a].def[buf[a].cur], buf[bb].vals, comp, flag, loOf(a));
      }
      checkLaunch();
    }
    if constexpr (!Comp::keepsUndefinedA) {
      Scope sc(this, "boolean_far");
      kPointwise2FarSign<T, Comp><<<grid1(nBricks), 256, 0, stream>>>(nBricks, buf[a].farSign,
                                                                      buf[bb].farSign, buf[a].farSign, comp);
      checkLaunch();
    }
    buf[a].bound = std::max(buf[a].bound, buf[bb].bound);
  }
  // BooleanOperation + Prune x2 (lsBooleanOperation.hpp:199-212)
  template <class Comp> void booleanOp(int a, int bb, Comp comp, int *flag = nullptr) {
    pointwise(a, bb, comp, flag);
    prunePair(a);
  }

  // An empty level set in buffer b (Domain(grid): positive everywhere, width 1).
  void clearBuffer(int b) {
    allocBuffers(b + 1);
    visitOk[b] = false;
    auto &B = buf[b];
    kFillSlots<T><<<blocksPass, 256, 0, stream>>>(slotList, nSlotsPtr(), B.vals, B.def[B.cur],
                                                  Lim<T>::max());
    checkLaunch();
    VLSG_CUDA(cudaMemsetAsync(B.farSign, 1, nBricks, stream));
    B.width = 1;
    B.bound = 0;
    B.nDef = 0;
    B.live = true;
  }
  // BooleanOperation INVERT on buffer b
  void invertBuffer(int b) {
    auto &B = buf[b];
    kNegateSlots<T><<<blocksPass, 256, 0, stream>>>(slotList, nSlotsPtr(), B.vals, B.farSign,
                                                    nBricks, loOf(b));
    checkLaunch();
  }

  // PrepareStencilLocalLaxFriedrichs (lsStencilLocalLaxFriedrichsScalar.hpp:
  // 423-477): the top level set becomes the inverted union of every depo
  // layer minus the first non-depo layer below it.  The reference tests a
  // layer with isDepo[isDepo[i]] (:448, it indexes the vector with the
  // element), which is kept.
  void prepareStencil(std::vector<bool> isDepo) {
    ++generation;
    pristine = false;
    loValid = false;
    pdTrack = pdSave = pdHas = false; // these operations carry no point data
    isDepo.resize(L, false);
    const int fin = L, above = L + 1;
    clearBuffer(fin);
    bool layerAboveIsDepo = false;
    int layer = L - 1;
    for (int i = L - 1; i >= 0; --i) {
      const size_t e = isDepo[i] ? 1 : 0;
      const bool depo = e < isDepo.size() && isDepo[e];
      if (depo) {
        if (!layerAboveIsDepo) {
          layer = i;
          layerAboveIsDepo = true;
        }
      } else {
        if (layerAboveIsDepo) {
          copyBuffer(layer, above);
          booleanOp(above, i, RelComplementComp<T>{});
          booleanOp(fin, above, MinComp<T>{});
          prune(fin, false);
        }
        layerAboveIsDepo = false;
      }
    }
    if (layerAboveIsDepo) booleanOp(fin, layer, MinComp<T>{});
    invertBuffer(fin);
    copyBuffer(fin, L - 1);
    buf[fin].live = false;
    if (above < 2 * L) buf[above].live = false;
    dropVisits();
    maintain();
    syncErr("PrepareStencilLocalLaxFriedrichs");
  }
  // FinalizeStencilLocalLaxFriedrichs (:480-492): top = INVERT(top) u the
  // level set below it.
  void finalizeStencil() {
    ++generation;
    pristine = false;
    loValid = false;
    pdTrack = pdSave = pdHas = false;
    dropVisits();
    invertBuffer(L - 1);
    booleanOp(L - 1, L - 2, MinComp<T>{});
    maintain();
    syncErr("FinalizeStencilLocalLaxFriedrichs");
  }

  void copyBuffer(int src, int dst) {
    allocBuffers(dst + 1);
    copyVisits(src, dst);
    auto &S = buf[src];
    auto &D = buf[dst];
    {
      Scope sc(this, "copy");
      kCopySlots16<T><<<blocksPass, 256, 0, stream>>>(slotList, nSlotsPtr(), S.vals, S.def[S.cur],
                                                      D.vals, D.def[D.cur], loOf(src), loOf(dst));
      checkLaunch();
    }
    VLSG_CUDA(cudaMemcpyAsync(D.farSign, S.farSign, nBricks, cudaMemcpyDeviceToDevice, stream));
    D.width = S.width;
    D.bound = S.bound;
    D.nDef = S.nDef;
    D.live = true;
  }

  // --------------------------------------------------------- one FE stage
  // integrateTime + findGlobalAlphas + reduceTimeStepHamiltonJacobi
  double computeRates(const vlsg_advect_params &P, double maxTimeStep) {
    const int top = L - 1;
    const int w = schemeWidth(P.spatial_scheme);
    if (w < 0) throw CudaError("Advect: Discretization scheme not found.", VLSG_ERR_ARGUMENT);
    expand(top, w); // prepareLS
    const int s = P.spatial_scheme;
    const bool globalLF = s == VLSG_LAX_FRIEDRICHS_1ST_ORDER || s == VLSG_LAX_FRIEDRICHS_2ND_ORDER;
    const bool lfFamily = !(s == VLSG_ENGQUIST_OSHER_1ST_ORDER || s == VLSG_ENGQUIST_OSHER_2ND_ORDER ||
                            s == VLSG_WENO_3RD_ORDER || s == VLSG_WENO_5TH_ORDER);
    double alphas[3] = {0, 0, 0};
    RateArgs<T> A{};
    A.g = g;
    A.m = mapView();
    for (int l = 0; l < L; ++l) A.ls[l] = view(l);
    A.L = L;
    A.slotList = slotList;
    A.nSlots = nSlotsPtr();
    A.nbr = nbr;
    A.cflag = cflag;
    A.def = buf[top].def[buf[top].cur];
    A.act = act;
    A.scheme = P.spatial_scheme;
    A.cfl = P.time_step_ratio;
    A.dissipationAlpha = P.dissipation_alpha;
    A.calcNormals = P.calculate_normal_vectors;
    A.adaptive = P.adaptive_time_stepping;
    A.adaptiveFactor = 1.0 / (P.adaptive_subdivisions < 1 ? 1u : P.adaptive_subdivisions);
    A.checkDiss = P.check_dissipation;
    A.minStep = scal;
    A.counts = rateCounts;
    A.err = errPtr();
    A.ownZ = ownAxis == 2;
    A.ownLo = (int)std::max<int64_t>(ownLo, INT_MIN / 2);
    A.ownHi = (int)std::min<int64_t>(ownHi, INT_MAX / 2);
    unsigned long long init[4] = {~0ull, 0, 0, 0};
    VLSG_CUDA(cudaMemcpyAsync(scal, init, sizeof(init), cudaMemcpyHostToDevice, stream));
    VLSG_CUDA(cudaMemsetAsync(rateCounts, 0, 2 * sizeof(unsigned long long), stream));
    if (globalLF) {
      A.alphaMax = scal + 1;
      if (velCb) gatherVelocities<1>(A);
      {
        Scope sc(this, "global_alphas");
        if (velCb) kRates<T, 1, true><<<blocksRate, RATE_THREADS, 0, stream>>>(A, vel);
        else kRates<T, 1><<<blocksRate, RATE_THREADS, 0, stream>>>(A, vel);
        checkLaunch();
      }
      VLSG_CUDA(cudaMemcpyAsync(pinScal, scal, sizeof(init), cudaMemcpyDeviceToHost, stream));
      VLSG_CUDA(cudaStreamSynchronize(stream));
      for (int k = 0; k < 3; ++k) {
        double a;
        std::memcpy(&a, &pinScal[1 + k], 8);
        alphas[k] = a;
      }
      reduceAcross(alphas, 3, VLSG_REDUCE_MAX); // findGlobalAlphas over all shards
      for (int k = 0; k < 3; ++k) A.globalAlpha[k] = T(alphas[k]);
      A.alphaMax = nullptr;
    } else if (lfFamily) {
      A.alphaMax = scal + 1;
    } else {
      A.alphaMax = nullptr;
    }
    const bool stencil = s == VLSG_STENCIL_LOCAL_LAX_FRIEDRICHS_1ST_ORDER;
    const int rateWarps = blocksRate * (RATE_THREADS / 32);
    if (stencil) {
      // the time-step alphas come from the last passing call (kSllfPick)
      A.alphaMax = nullptr;
      A.sllfEps = std::cbrt(std::numeric_limits<double>::epsilon());
      A.maxDissipation = P.max_dissipation > 0 ? P.max_dissipation : DBL_MAX;
      A.sllfKey = scratch<unsigned long long>(X_SKEY, rateWarps);
      A.sllfAlpha = scratch<double>(X_SALPHA, 3 * (size_t)rateWarps);
    }
    A.voidMask = P.ignore_voids ? markVoids() : nullptr;
    if (velCb) gatherVelocities<0>(A);
    if (!rateCap) ensureRateCap(65536);
    for (;;) {
    // the compact rate arrays; a pass that finds them too small is run again
    // with larger ones (the bricks left out wrote nothing)
    A.rateV = rateV;
    A.rateStop = rateStop;
    A.rateD = pdSave ? rateD : nullptr;
    A.rateLen = rateLen;
    A.rateCap = rateCap;
    A.rateNext = rateCounts + 2;
    A.rateBase = rateBase;
    VLSG_CUDA(cudaMemsetAsync(rateCounts + 2, 0, sizeof(unsigned long long), stream));
    {
      // stencil input (each band value once) + output per active point
      Scope sc(this, "rates", [this] {
        lastActive = (int64_t)readU64(rateCounts + 0);
        lastBand = (int64_t)readU64(rateCounts + 1);
        return double(sizeof(T)) * double(lastBand + lastActive);
      });
      const bool weno = s == VLSG_WENO_3RD_ORDER || s == VLSG_WENO_5TH_ORDER;
      if (stencil) {
        if (velCb) kRates<T, 0, true, FAM_STENCIL><<<blocksRate, RATE_THREADS, 0, stream>>>(A, vel);
        else kRates<T, 0, false, FAM_STENCIL><<<blocksRate, RATE_THREADS, 0, stream>>>(A, vel);
        checkLaunch();
        kSllfPick<<<1, 1024, 0, stream>>>(A.sllfKey, A.sllfAlpha, rateWarps, scal + 1);
      } else if (weno) {
        if (velCb) kRates<T, 0, true, FAM_WENO><<<blocksRateWeno, RATE_THREADS, 0, stream>>>(A, vel);
        else kRates<T, 0, false, FAM_WENO><<<blocksRateWeno, RATE_THREADS, 0, stream>>>(A, vel);
      } else if (velCb) {
        kRates<T, 0, true><<<blocksRate, RATE_THREADS, 0, stream>>>(A, vel);
      } else {
        kRates<T, 0><<<blocksRate, RATE_THREADS, 0, stream>>>(A, vel);
      }
      checkLaunch();
    }
    VLSG_CUDA(cudaMemcpyAsync(pinScal, scal, sizeof(init), cudaMemcpyDeviceToHost, stream));
    VLSG_CUDA(cudaMemcpyAsync(pinScal + 4, rateCounts, 3 * sizeof(unsigned long long),
                              cudaMemcpyDeviceToHost, stream));
    syncErr("rates");
    const unsigned long long need = pinScal[6];
    if (need <= rateCap) break;
    ensureRateCap(need + need / 4 + 4096);
    VLSG_CUDA(cudaMemcpyAsync(scal, init, sizeof(init), cudaMemcpyHostToDevice, stream));
    VLSG_CUDA(cudaMemsetAsync(rateCounts, 0, 2 * sizeof(unsigned long long), stream));
    }
    std::memcpy(hScal, pinScal, sizeof(hScal));
    lastActive = (int64_t)pinScal[4];
    lastBand = (int64_t)pinScal[5];
    pointUpdates += (uint64_t)lastActive;
    double tempMax = maxTimeStep;
    double m = DBL_MAX; // no active point: no bound from the points
    if (hScal[0] != ~0ull) std::memcpy(&m, &hScal[0], 8);
    reduceAcross(&m, 1, VLSG_REDUCE_MIN); // the time step over all shards
    if (m < tempMax) tempMax = m;
    if (lfFamily) {
      double fa[3];
      if (globalLF) {
        for (int k = 0; k < 3; ++k) fa[k] = alphas[k];
      } else {
        for (int k = 0; k < 3; ++k) std::memcpy(&fa[k], &hScal[1 + k], 8);
        if (!stencil) reduceAcross(fa, 3, VLSG_REDUCE_MAX);
      }
      double timeStep = 0;
      for (int i = 0; i < 3; ++i) timeStep += fa[i] / g.delta;
      timeStep = 1.0 / timeStep;
      tempMax = (tempMax < timeStep) ? tempMax : timeStep;
    }
    if (tempMax < maxTimeStep) maxTimeStep = tempMax;
    currentTimeStep = maxTimeStep;
    return maxTimeStep;
  }

  // setIgnoreVoids: MarkVoidPoints on the top level set (vlsg_voids.cuh);
  // returns the void bits per slot.
  const uint64_t *markVoids() {
    Scope sc(this, "mark_voids");
    const int top = L - 1;
    const size_t nodes = poolCells + (size_t)nBricks;
    if (nodes >= (size_t)UINT32_MAX)
      throw CudaError("setIgnoreVoids: too many cells for the void search", VLSG_ERR_CAPACITY);
    uint32_t *parent = scratch<uint32_t>(X_VPARENT, nodes);
    uint64_t *mask = scratch<uint64_t>(X_VMASK, (size_t)capSlots * 8);
    uint32_t *topNode = scratch<uint32_t>(X_VTOP, 2);
    const Buf<T> b = view(top);
    kVoidInit<<<grid1(nodes), 256, 0, stream>>>(parent, nodes);
    kVoidUnionCells<T><<<blocksPass, 256, 0, stream>>>(g, mapView(), b, slotList, nSlotsPtr(),
                                                       poolCells, parent, errPtr());
    kVoidUnionBricks<T><<<grid1(nBricks), 256, 0, stream>>>(g, mapView(), b, nBricks, poolCells,
                                                            parent, errPtr());
    kVoidTop<T><<<1, 32, 0, stream>>>(g, mapView(), b, poolCells, parent, topNode, errPtr());
    VLSG_CUDA(cudaMemsetAsync(mask, 0, (size_t)capSlots * 8 * sizeof(uint64_t), stream));
    kVoidMark<T><<<blocksPass, 256, 0, stream>>>(g, mapView(), b, slotList, nSlotsPtr(),
                                                 buf[top].def[buf[top].cur], poolCells, parent,
                                                 topNode, mask, errPtr());
    checkLaunch();
    syncErr("MarkVoidPoints");
    return mask;
  }

  // Host callback mode: the queries of rate pass MODE (every active point x
  // material x site), answered by the callback from a pool of host threads,
  // become A's velocity table.
  template <int MODE> void gatherVelocities(RateArgs<T> &A) {
    Scope sc(this, "velocity_callback");
    const int top = L - 1;
    const int nList = readI32(nSlotsPtr());
    uint32_t *cnt = scratch<uint32_t>(X_VCNT, nList);
    uint32_t *off = scratch<uint32_t>(X_VOFF, nList);
    uint32_t *sums = scratch<uint32_t>(X_VSUMS, scanScratch((size_t)nList) + 64);
    kActiveCount<T><<<blocksRate, RATE_THREADS, 0, stream>>>(A, cnt);
    checkLaunch();
    scanExclusive(cnt, off, nList, sums);
    const size_t nAct = scanTotal(sums, nList);
    const int sites = velocitySites(A.scheme, MODE);
    const size_t nQ = nAct * (size_t)L * sites;
    if (nQ > ((size_t)1 << 28))
      throw CudaError("velocity callback: more than 2^28 queries in one rate pass",
                      VLSG_ERR_CAPACITY);
    xBuf = -1; // the point layout below reuses the exchange's scratch
    pointLayout(top, nList);
    const PointRanks R{slotBrick, (const uint32_t *)xs[X_POS].p, (const int4 *)xs[X_BOUNDS].p,
                       (const uint32_t *)xs[X_P].p, buf[top].def[buf[top].cur]};
    double *qc = scratch<double>(X_QC, 3 * nQ);
    int32_t *qm = scratch<int32_t>(X_QM, nQ);
    double *qn = scratch<double>(X_QN, 3 * nQ);
    uint64_t *qp = scratch<uint64_t>(X_QP, nQ);
    double *vs = scratch<double>(X_VS, nQ);
    double *vv = scratch<double>(X_VV, 3 * nQ);
    A.actOff = off;
    A.velS = vs;
    A.velV = vv;
    A.velSites = sites;
    A.alphaTab = nullptr;
    A.velS2 = nullptr;
    if (!nQ) return;
    kVelGather<T, MODE><<<blocksRate, RATE_THREADS, 0, stream>>>(A, R, sites, qc, qm, qn, qp);
    checkLaunch();
    askVelocity(nQ, qc, qm, qn, qp, vs, vv);
    if (MODE == 0 && A.scheme == VLSG_LOCAL_LAX_FRIEDRICHS_ANALYTICAL_1ST_ORDER && alphaCb)
      gatherAlphas(A, nAct);
    if (MODE == 0 && A.scheme == VLSG_STENCIL_LOCAL_LAX_FRIEDRICHS_1ST_ORDER) {
      // second round: the nudged normals, which depend on the first answers
      const size_t n2 = nAct * (size_t)L * 162;
      if (n2 > ((size_t)1 << 28))
        throw CudaError("velocity callback: more than 2^28 queries in one rate pass",
                        VLSG_ERR_CAPACITY);
      double *qc2 = scratch<double>(X_QC2, 3 * n2);
      double *qn2 = scratch<double>(X_QN2, 3 * n2);
      int32_t *qm2 = scratch<int32_t>(X_QM2, n2);
      uint64_t *qp2 = scratch<uint64_t>(X_QP2, n2);
      double *vs2 = scratch<double>(X_VS2, n2);
      kStencilGather<T><<<blocksRate, RATE_THREADS, 0, stream>>>(A, R, qc2, qm2, qn2, qp2);
      checkLaunch();
      askVelocity(n2, qc2, qm2, qn2, qp2, vs2, nullptr);
      A.velS2 = vs2;
    }
  }

  // The velocity callback on n queries staged on the device; the scalar (and,
  // with vOut, the vector) answers land in device arrays, stream-ordered.
  void askVelocity(size_t n, const double *qc, const int32_t *qm, const double *qn,
                   const uint64_t *qp, double *sOut, double *vOut) {
    // earlier copies out of the pinned staging buffers are complete
    VLSG_CUDA(cudaStreamSynchronize(stream));
    double *hc = pinned<double>(H_QC, 3 * n);
    int32_t *hm = pinned<int32_t>(H_QM, n);
    double *hn = pinned<double>(H_QN, 3 * n);
    uint64_t *hp = pinned<uint64_t>(H_QP, n);
    double *hsv = pinned<double>(H_VS, n);
    double *hvv = pinned<double>(H_VV, 3 * n);
    VLSG_CUDA(cudaMemcpyAsync(hc, qc, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, stream));
    VLSG_CUDA(cudaMemcpyAsync(hm, qm, n * sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
    VLSG_CUDA(cudaMemcpyAsync(hn, qn, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, stream));
    VLSG_CUDA(cudaMemcpyAsync(hp, qp, n * sizeof(uint64_t), cudaMemcpyDeviceToHost, stream));
    syncErr("velocity queries");
    if (g.planar) {
      // D = 2: the queries the gathers marked with material -1 (sites off
      // the plane) are not asked; their answers are 0 and nothing reads them
      std::vector<size_t> at;
      at.reserve(n);
      for (size_t i = 0; i < n; ++i)
        if (hm[i] >= 0) at.push_back(i);
      const size_t k = at.size();
      std::vector<double> qc(3 * k), qn(3 * k), qs(k), qv(3 * k);
      std::vector<int32_t> qm(k);
      std::vector<uint64_t> qp(k);
      for (size_t j = 0; j < k; ++j) {
        const size_t i = at[j];
        for (int d = 0; d < 3; ++d) qc[3 * j + d] = hc[3 * i + d], qn[3 * j + d] = hn[3 * i + d];
        qm[j] = hm[i], qp[j] = hp[i];
      }
      hostPool(k, [&](size_t i, int64_t m) {
        return velCb(velUser, m, qc.data() + 3 * i, qm.data() + i, qn.data() + 3 * i,
                     qp.data() + i, qs.data() + i, qv.data() + 3 * i);
      }, "the velocity callback returned ");
      std::fill(hsv, hsv + n, 0.0);
      std::fill(hvv, hvv + 3 * n, 0.0);
      for (size_t j = 0; j < k; ++j) {
        hsv[at[j]] = qs[j];
        for (int d = 0; d < 3; ++d) hvv[3 * at[j] + d] = qv[3 * j + d];
      }
    } else {
      hostPool(n, [&](size_t i, int64_t m) {
        return velCb(velUser, m, hc + 3 * i, hm + i, hn + 3 * i, hp + i, hsv + i, hvv + 3 * i);
      }, "the velocity callback returned ");
    }
    VLSG_CUDA(cudaMemcpyAsync(sOut, hsv, n * sizeof(double), cudaMemcpyHostToDevice, stream));
    if (vOut)
      VLSG_CUDA(cudaMemcpyAsync(vOut, hvv, 3 * n * sizeof(double), cudaMemcpyHostToDevice, stream));
  }

  // LocalLaxFriedrichsAnalytical with host callbacks: every active point x
  // material x box neighbour x direction asked through the alpha callback.
  void gatherAlphas(RateArgs<T> &A, size_t nAct) {
    const size_t nA = nAct * (size_t)L * 81;
    if (nA > ((size_t)1 << 28))
      throw CudaError("alpha callback: more than 2^28 queries in one rate pass", VLSG_ERR_CAPACITY);
    int32_t *ad = scratch<int32_t>(X_AD, nA);
    int32_t *am = scratch<int32_t>(X_AM, nA);
    double *ac = scratch<double>(X_AC, 3 * nA);
    double *av = scratch<double>(X_AV, nA);
    kAlphaGather<T><<<blocksRate, RATE_THREADS, 0, stream>>>(A, ad, am, ac);
    checkLaunch();
    VLSG_CUDA(cudaStreamSynchronize(stream));
    int32_t *hd = pinned<int32_t>(H_AD, nA);
    int32_t *hm = pinned<int32_t>(H_AM, nA);
    double *hc = pinned<double>(H_AC, 3 * nA);
    double *hv = pinned<double>(H_AV, nA);
    VLSG_CUDA(cudaMemcpyAsync(hd, ad, nA * sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
    VLSG_CUDA(cudaMemcpyAsync(hm, am, nA * sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
    VLSG_CUDA(cudaMemcpyAsync(hc, ac, 3 * nA * sizeof(double), cudaMemcpyDeviceToHost, stream));
    syncErr("alpha queries");
    if (g.planar) {
      // D = 2: only the plane's 9 box neighbours (q 9..17) and the directions
      // x and y are asked, as the 2D reference asks them; the rate kernel
      // reads no other entry
      const size_t nq = nA / 81 * 18;
      std::vector<size_t> at(nq);
      std::vector<int32_t> qd(nq), qm(nq);
      std::vector<double> qc(3 * nq), qv(nq);
      size_t k = 0;
      for (size_t e = 0; e < nA; ++e) {
        const size_t q = (e / 3) % 27;
        if (q < 9 || q >= 18 || e % 3 == 2) continue;
        at[k] = e, qd[k] = hd[e], qm[k] = hm[e];
        for (int c = 0; c < 3; ++c) qc[3 * k + c] = hc[3 * e + c];
        ++k;
      }
      hostPool(nq, [&](size_t i, int64_t n) {
        return alphaCb(alphaUser, n, qd.data() + i, qm.data() + i, qc.data() + 3 * i, qv.data() + i);
      }, "the dissipation alpha callback returned ");
      std::fill(hv, hv + nA, 0.0);
      for (size_t i = 0; i < nq; ++i) hv[at[i]] = qv[i];
    } else {
      hostPool(nA, [&](size_t i, int64_t n) {
        return alphaCb(alphaUser, n, hd + i, hm + i, hc + 3 * i, hv + i);
      }, "the dissipation alpha callback returned ");
    }
    VLSG_CUDA(cudaMemcpyAsync(av, hv, nA * sizeof(double), cudaMemcpyHostToDevice, stream));
    A.alphaTab = av;
  }

  // Runs fn(first, count) over [0, n) in chunks of 4096 from a pool of host
  // threads; a non-zero return ends the work with VLSG_ERR_CALLBACK.
  template <class Fn> void hostPool(size_t n, Fn fn, const char *what) {
    const size_t chunk = 4096;
    const unsigned hw = std::thread::hardware_concurrency();
    const int nt = (int)std::min<size_t>(std::max(1u, std::min(hw, 64u)), (n + chunk - 1) / chunk);
    std::atomic<size_t> next{0};
    std::atomic<int> failed{0};
    auto worker = [&] {
      for (size_t i = next.fetch_add(chunk); i < n && !failed.load(); i = next.fetch_add(chunk)) {
        const int rc = fn(i, (int64_t)std::min(chunk, n - i));
        if (rc != 0) {
          int zero = 0;
          failed.compare_exchange_strong(zero, rc);
        }
      }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back(worker);
    worker();
    for (auto &th : pool) th.join();
    if (failed) throw CudaError(std::string(what) + std::to_string(failed.load()), VLSG_ERR_CALLBACK);
  }

  void adjustLowerLayers(const vlsg_advect_params &P) {
    if (P.spatial_scheme == VLSG_STENCIL_LOCAL_LAX_FRIEDRICHS_1ST_ORDER) return;
    for (int i = 0; i + 1 < L; ++i) booleanOp(i, L - 1, MaxComp<T>{});
  }

  double evolveForwardEuler(const vlsg_advect_params &P, double maxTimeStep,
                            bool updateLowerLayers) {
    const double dt = computeRates(P, maxTimeStep);
    updateRebuild(dt);
    if (!deferMaintain) maintain();
    if (updateLowerLayers) adjustLowerLayers(P);
    return dt;
  }
  // Within an RK step with time_step_ratio <= 0.5 a stage moves the surface
  // by at most half a cell, and no band is wider than 4.5 cells on either
  // side (LocalLaxFriedrichs 2nd order): every cell the step defines lies
  // within 7 cells of a cell defined at the step's start, inside the brick
  // margin the last maintenance left.  Such steps maintain once, at the end;
  // the device check (band reached an unallocated brick) stays armed.
  bool deferMaintain = false;

  bool combineLevelSets(const vlsg_advect_params &P, double wTarget, double wSource) {
    int steps = 1;
    if (P.temporal_scheme == VLSG_RUNGE_KUTTA_2ND_ORDER) steps = 2;
    else if (P.temporal_scheme == VLSG_RUNGE_KUTTA_3RD_ORDER) steps = 3;
    const int expansionWidth = (int)std::ceil(2.0 * steps * P.time_step_ratio + 1);
    const int top = L - 1, init = 2 * L - 1;
    expand(top, expansionWidth);
    expand(init, expansionWidth);
    VLSG_CUDA(cudaMemsetAsync(flagPtr(), 0, sizeof(int), stream));
    CombineComp<T> comp{wTarget, wSource};
    pointwise(top, init, comp, flagPtr());
    prunePair(top);
    rebuild(top);
    if (!deferMaintain) maintain();
    if (L > 1) {
      VLSG_CUDA(cudaMemcpyAsync(pinCounters, counters, 16 * sizeof(int), cudaMemcpyDeviceToHost, stream));
      VLSG_CUDA(cudaStreamSynchronize(stream));
      double moved = pinCounters[4] != 0 ? 1.0 : 0.0;
      reduceAcross(&moved, 1, VLSG_REDUCE_MAX);
      return moved != 0.0;
    }
    return false;
  }

  // The cross-shard reduction (vlsg_set_reduction_callback), or nothing.
  void reduceAcross(double *v, int n, int op) {
    if (!reduceCb) return;
    const int rc = reduceCb(reduceUser, v, n, op);
    if (rc != 0)
      throw CudaError("the reduction callback returned " + std::to_string(rc), VLSG_ERR_CALLBACK);
  }

  // The RK copy of the top level set is first read by the stage combination,
  // after Expand to E = ceil(2 steps ratio + 1) (combineLevelSets).  When the
  // first stage's Expand to the scheme's width S and the copy's Expand to E
  // both only define new cells (|value| <= min(E, S) / 2 on the defined
  // cells), each of their cycles depends only on the width it starts from,
  // so the first stage's band at width min(E, S) is the copy expanded to that
  // width, value for value.  The copy is taken there (expand()), which saves
  // the copy's own Expand cycles.  Otherwise it is taken now.
  int saveTopAt = 0;
  void saveTop(const vlsg_advect_params &P, int steps) {
    const int top = L - 1;
    const int E = (int)std::ceil(2.0 * steps * P.time_step_ratio + 1);
    const int S = schemeWidth(P.spatial_scheme);
    const int at = std::min(E, S);
    saveTopAt = 0;
    if (S < 0 || buf[top].width >= at || buf[top].bound > 0.5 * at) copyBuffer(top, L + top);
    else saveTopAt = at;
  }
  void restoreLower() {
    for (int l = 0; l + 1 < L; ++l) {
      copyVisits(L + l, l);
      // copy initial back into the current buffer
      auto &S = buf[L + l];
      auto &D = buf[l];
      {
        Scope sc(this, "copy");
        kCopySlots16<T><<<blocksPass, 256, 0, stream>>>(slotList, nSlotsPtr(), S.vals,
                                                        S.def[S.cur], D.vals, D.def[D.cur],
                                                        loOf(L + l), loOf(l));
        checkLaunch();
      }
      VLSG_CUDA(cudaMemcpyAsync(D.farSign, S.farSign, nBricks, cudaMemcpyDeviceToDevice, stream));
      D.width = S.width;
      D.bound = S.bound;
      D.nDef = S.nDef;
    }
  }

  // velocityUpdateCallback with the top level set in the exchange format
  void callUpdate() {
    ++generation; // the level sets changed since the last exchange
    const int top = L - 1;
    const int64_t n = compact(top, nullptr, nullptr, 0);
    std::vector<int32_t> idx(3 * (size_t)n);
    std::vector<double> val((size_t)n);
    compact(top, idx.data(), val.data(), n);
    const int64_t m = runs(top, nullptr, nullptr, 0);
    std::vector<int32_t> rs(3 * (size_t)m);
    std::vector<int8_t> sg((size_t)m);
    runs(top, rs.data(), sg.data(), m);
    const vlsg_levelset_view v{n, idx.data(), val.data(), m, rs.data(), sg.data(), buf[top].width};
    const int rc = updCb(updUser, &v);
    if (rc != 0)
      throw CudaError("the velocity update callback returned " + std::to_string(rc),
                      VLSG_ERR_CALLBACK);
  }

  // Heun RK2 (lsAdvectIntegrationSchemes.hpp:59-108): with a velocity-update
  // callback, stage 1 adjusts the lower layers, the callback runs after it,
  // and the lower layers are restored when the combination etched.
  // the deferred maintenance at the end of an RK step
  void endStep() {
    if (deferMaintain) {
      deferMaintain = false;
      maintain();
    }
  }

  double evolveRungeKutta2(const vlsg_advect_params &P, double maxTimeStep) {
    const bool cb = updCb != nullptr;
    deferMaintain = P.time_step_ratio <= 0.5;
    if (cb)
      for (int l = 0; l + 1 < L; ++l) copyBuffer(l, L + l);
    saveTop(P, 2);
    const double dt1 = evolveForwardEuler(P, maxTimeStep, cb);
    if (dt1 <= 0.) {
      endStep();
      return 0.;
    }
    if (cb) callUpdate();
    const double dt2 = evolveForwardEuler(P, dt1, false);
    const bool etched = combineLevelSets(P, 0.5, 0.5);
    if (etched && cb) restoreLower();
    adjustLowerLayers(P);
    endStep();
    return 0.5 * dt1 + 0.5 * dt2;
  }
  // SSP RK3 (:110-168)
  double evolveRungeKutta3(const vlsg_advect_params &P, double maxTimeStep) {
    const bool cb = updCb != nullptr;
    deferMaintain = P.time_step_ratio <= 0.5;
    for (int l = 0; l + 1 < L; ++l) copyBuffer(l, L + l);
    saveTop(P, 3);
    const double dt1 = evolveForwardEuler(P, maxTimeStep, cb);
    if (dt1 <= 0.) {
      endStep();
      return 0.;
    }
    if (cb) callUpdate();
    const double dt2 = evolveForwardEuler(P, dt1, false);
    const bool etched1 = combineLevelSets(P, 0.75, 0.25);
    if (etched1 && cb) restoreLower();
    adjustLowerLayers(P);
    if (cb) callUpdate();
    const double dt3 = evolveForwardEuler(P, dt1, false);
    const bool etched2 = combineLevelSets(P, 1.0 / 3.0, 2.0 / 3.0);
    if (etched2) restoreLower();
    adjustLowerLayers(P);
    endStep();
    return (dt1 + dt2 + 4.0 * dt3) / 6.0;
  }
  double advect(const vlsg_advect_params &P, double maxTimeStep) {
    switch (P.temporal_scheme) {
    case VLSG_RUNGE_KUTTA_2ND_ORDER: return evolveRungeKutta2(P, maxTimeStep);
    case VLSG_RUNGE_KUTTA_3RD_ORDER: return evolveRungeKutta3(P, maxTimeStep);
    default: return evolveForwardEuler(P, maxTimeStep, true);
    }
  }

  void apply(const vlsg_advect_params &P, vlsg_advect_result &r) override {
    ++generation;
    deferMaintain = false; // an earlier apply may have ended in an error mid-step
    saveTopAt = 0;
    // point data: every apply ends with a rebuild of the top level set, which
    // keeps it only with updatePointData (lsAdvect.hpp:418-423)
    const bool wantPd = P.track_point_data || P.save_advection_velocities;
    pdTrack = wantPd && P.update_point_data;
    pdSave = pdTrack && P.save_advection_velocities;
    pdHas = false;
    if (pdTrack) initPointData();
    // FP32 compensation terms for this advection (fp32_compensation)
    compActive = kComp && P.fp32_compensation != 0;
    if (compActive && !loValid) {
      // the RK copy takes its terms from the top level set: the part of the
      // uploaded doubles the floats dropped, or zero
      loWanted = true;
      allocBuffers(L);
      VLSG_CUDA(cudaMemsetAsync(buf[L - 1].lo, 0, buf[L - 1].capLo * BV * sizeof(float), stream));
      if (pristine && upN) {
        kScatterLo<T><<<grid1(upN), 256, 0, stream>>>(g, (int)upN, upIdx, upVals, brickMap,
                                                      buf[L - 1].lo);
        checkLaunch();
      }
    }
    loValid = compActive; // without compensation the passes leave the terms stale
    pristine = false;
    const bool sllf = P.spatial_scheme == VLSG_STENCIL_LOCAL_LAX_FRIEDRICHS_1ST_ORDER;
    rebuildCutoff = sllf ? 1.5 : 1.0;
    rebuildWidth = sllf ? 3 : 2;
    pointUpdates = 0;
    stages = 0;
    const uint64_t l0 = launches;
    double advectedTime = 0.;
    unsigned steps = 0;
    const uint32_t maxSteps = P.max_steps ? P.max_steps : 10000000u;
    if (P.advection_time == 0.) {
      advectedTime = advect(P, std::numeric_limits<double>::max());
      steps = 1;
    } else {
      double currentTime = 0.0;
      while (currentTime < P.advection_time) {
        currentTime += advect(P, P.advection_time - currentTime);
        ++steps;
        if (P.single_step) break;
        if (steps >= maxSteps) throw CudaError("step limit reached", VLSG_ERR_NUMERIC);
      }
      advectedTime = currentTime;
    }
    syncErr("advect");
    compActive = false;
    pdHas = pdTrack;
    pdTrack = pdSave = false;
    r.advected_time = advectedTime;
    r.current_time_step = currentTimeStep;
    r.number_of_time_steps = steps;
    r.number_of_stages = stages;
    r.point_updates = pointUpdates;
    r.kernel_launches = launches - l0;
  }

  // ------------------------------------------------------- batching form
  // Many independent domains in one brick box (GridDev's domain table): one
  // launch per pass and per rate / update step over the bricks of all
  // domains, the time step of every domain on the device (kDomainSteps), no
  // host synchronisation inside the step.
  int nDom = 0;
  DomainDev *domDev = nullptr;
  int *domOfBzDev = nullptr;
  double *domDelta = nullptr;
  vlsg_velocity_desc *domVelDev = nullptr;
  unsigned long long *domRed = nullptr;     // RED_WORDS per domain (vlsg_rates.cuh)
  unsigned long long *domRedInit = nullptr; // their reset values
  unsigned long long *domUpdates = nullptr; // point updates of the step per domain
  double *domDt = nullptr;                  // stage steps a, b, c and advected time

  void buildBatch(const GridDev &grid, const std::vector<DomainDev> &doms,
                  const std::vector<int> &domOfBz, const std::vector<double> &delta,
                  const std::vector<vlsg_velocity_desc> &vels, std::vector<StagedLS> &ls) override {
    ensureSmall();
    auto f = [](void *p) { if (p) cudaFree(p); };
    f(domDev); f(domOfBzDev); f(domDelta); f(domVelDev); f(domRed); f(domUpdates); f(domDt);
    f(domRedInit);
    nDom = (int)doms.size();
    rateShape[0] = rateShape[1] = 0; // tune again for the new batch
    VLSG_CUDA(cudaMalloc(&domDev, nDom * sizeof(DomainDev)));
    VLSG_CUDA(cudaMalloc(&domOfBzDev, domOfBz.size() * sizeof(int)));
    VLSG_CUDA(cudaMalloc(&domDelta, nDom * sizeof(double)));
    VLSG_CUDA(cudaMalloc(&domVelDev, nDom * sizeof(vlsg_velocity_desc)));
    VLSG_CUDA(cudaMalloc(&domRed, (size_t)RED_WORDS * nDom * sizeof(unsigned long long)));
    VLSG_CUDA(cudaMalloc(&domRedInit, (size_t)RED_WORDS * nDom * sizeof(unsigned long long)));
    VLSG_CUDA(cudaMalloc(&domUpdates, nDom * sizeof(unsigned long long)));
    VLSG_CUDA(cudaMalloc(&domDt, 4 * (size_t)nDom * sizeof(double)));
    VLSG_CUDA(cudaMemcpyAsync(domDev, doms.data(), nDom * sizeof(DomainDev), cudaMemcpyHostToDevice, stream));
    VLSG_CUDA(cudaMemcpyAsync(domOfBzDev, domOfBz.data(), domOfBz.size() * sizeof(int),
                              cudaMemcpyHostToDevice, stream));
    VLSG_CUDA(cudaMemcpyAsync(domDelta, delta.data(), nDom * sizeof(double), cudaMemcpyHostToDevice, stream));
    VLSG_CUDA(cudaMemcpyAsync(domVelDev, vels.data(), nDom * sizeof(vlsg_velocity_desc),
                              cudaMemcpyHostToDevice, stream));
    std::vector<unsigned long long> red((size_t)RED_WORDS * nDom, 0ull);
    for (int d = 0; d < nDom; ++d) red[(size_t)RED_WORDS * d + RED_MIN] = ~0ull;
    VLSG_CUDA(cudaMemcpyAsync(domRed, red.data(), red.size() * sizeof(unsigned long long),
                              cudaMemcpyHostToDevice, stream));
    VLSG_CUDA(cudaMemcpyAsync(domRedInit, red.data(), red.size() * sizeof(unsigned long long),
                              cudaMemcpyHostToDevice, stream));
    VLSG_CUDA(cudaStreamSynchronize(stream)); // the host vectors go out of scope
    GridDev g2 = grid;
    g2.nDom = nDom;
    g2.dom = domDev;
    g2.domOfBz = domOfBzDev;
    build(g2, ls, 0);
  }

  // Launch-shape autotuner of the batching form.  The rate kernel is
  // compiled for several resident-block counts per SM (FP32: 2, 3 or 4, i.e.
  // up to 128, 80 or 64 registers per thread; FP64: 1 or 2): more blocks hide
  // more latency, fewer spill less.  The first stage of the first batch step
  // runs every shape once (the pass only reads the level sets, so it can run
  // again; its reductions are reset in between) and keeps the fastest per
  // scheme family (WENO or not) until the batch changes.
  int rateShape[2] = {0, 0};
  bool capturing = false;
  static const char *rateShapeName(int k) {
    switch (k) {
    case 1: return "rates_b1";
    case 2: return "rates_b2";
    case 3: return "rates_b3";
    default: return "rates_b4";
    }
  }
  void launchBatchRates(const RateArgs<T> &A, bool weno, int k) {
    const dim3 grid(numSMs * k);
    if constexpr (sizeof(T) == 4) {
      if (weno) {
        if (k == 2) kRates<T, 0, false, FAM_WENO, true, 2><<<grid, RATE_THREADS, 0, stream>>>(A, vel);
        else if (k == 3) kRates<T, 0, false, FAM_WENO, true, 3><<<grid, RATE_THREADS, 0, stream>>>(A, vel);
        else kRates<T, 0, false, FAM_WENO, true, 4><<<grid, RATE_THREADS, 0, stream>>>(A, vel);
      } else {
        if (k == 2) kRates<T, 0, false, FAM_ANY, true, 2><<<grid, RATE_THREADS, 0, stream>>>(A, vel);
        else if (k == 3) kRates<T, 0, false, FAM_ANY, true, 3><<<grid, RATE_THREADS, 0, stream>>>(A, vel);
        else kRates<T, 0, false, FAM_ANY, true, 4><<<grid, RATE_THREADS, 0, stream>>>(A, vel);
      }
    } else {
      if (weno) {
        if (k == 1) kRates<T, 0, false, FAM_WENO, true, 1><<<grid, RATE_THREADS, 0, stream>>>(A, vel);
        else kRates<T, 0, false, FAM_WENO, true, 2><<<grid, RATE_THREADS, 0, stream>>>(A, vel);
      } else {
        if (k == 1) kRates<T, 0, false, FAM_ANY, true, 1><<<grid, RATE_THREADS, 0, stream>>>(A, vel);
        else kRates<T, 0, false, FAM_ANY, true, 2><<<grid, RATE_THREADS, 0, stream>>>(A, vel);
      }
    }
  }
  void tuneRates(const RateArgs<T> &A, bool weno) {
    const std::vector<int> shapes = sizeof(T) == 4 ? std::vector<int>{2, 3, 4} : std::vector<int>{1, 2};
    cudaEvent_t e0, e1;
    VLSG_CUDA(cudaEventCreate(&e0));
    VLSG_CUDA(cudaEventCreate(&e1));
    float best = 0.f;
    int pick = shapes.back();
    for (int k : shapes) {
      VLSG_CUDA(cudaMemsetAsync(rateCounts + 2, 0, sizeof(unsigned long long), stream));
      VLSG_CUDA(cudaEventRecord(e0, stream));
      launchBatchRates(A, weno, k);
      checkLaunch();
      VLSG_CUDA(cudaEventRecord(e1, stream));
      VLSG_CUDA(cudaEventSynchronize(e1));
      float ms = 0.f;
      VLSG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      if (k == shapes.front() || ms < best) best = ms, pick = k;
      // the next run (and the real one) starts from fresh reductions
      VLSG_CUDA(cudaMemcpyAsync(domRed, domRedInit, (size_t)RED_WORDS * nDom * sizeof(unsigned long long),
                                cudaMemcpyDeviceToDevice, stream));
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    rateShape[weno ? 1 : 0] = pick;
  }

  // One forward-Euler stage of every domain: Expand, rates with per-domain
  // reductions, the per-domain step (capped by cap, null: none) into out,
  // value update, Reduce + rebuild.
  void stageBatch(const vlsg_advect_params &P, const double *cap, double *out, bool first) {
    const int top = L - 1;
    expand(top, schemeWidth(P.spatial_scheme));
    const int s = P.spatial_scheme;
    const bool lfFamily = !(s == VLSG_ENGQUIST_OSHER_1ST_ORDER || s == VLSG_ENGQUIST_OSHER_2ND_ORDER ||
                            s == VLSG_WENO_3RD_ORDER || s == VLSG_WENO_5TH_ORDER);
    RateArgs<T> A{};
    A.g = g;
    A.m = mapView();
    for (int l = 0; l < L; ++l) A.ls[l] = view(l);
    A.L = L;
    A.slotList = slotList;
    A.nSlots = nSlotsPtr();
    A.nbr = nbr;
    A.cflag = cflag;
    A.def = buf[top].def[buf[top].cur];
    A.act = act;
    A.scheme = s;
    A.cfl = P.time_step_ratio;
    A.dissipationAlpha = P.dissipation_alpha;
    A.calcNormals = P.calculate_normal_vectors;
    A.adaptive = P.adaptive_time_stepping;
    A.adaptiveFactor = 1.0 / (P.adaptive_subdivisions < 1 ? 1u : P.adaptive_subdivisions);
    A.checkDiss = P.check_dissipation;
    A.rateV = rateV;
    A.rateStop = rateStop;
    A.rateLen = rateLen;
    A.rateCap = rateCap;
    A.rateNext = rateCounts + 2;
    A.rateBase = rateBase;
    A.rateOverflowErr = 1024; // capacity is set before the step (applyBatch)
    A.err = errPtr();
    A.slotDom = slotDom;
    A.domDelta = domDelta;
    A.domVel = domVelDev;
    A.domRed = domRed;
    const bool weno = s == VLSG_WENO_3RD_ORDER || s == VLSG_WENO_5TH_ORDER;
    const int fi = weno ? 1 : 0;
    if (!rateShape[fi] && !capturing) tuneRates(A, weno);
    // untuned (a family first met while capturing): the single-domain shape
    const int shape = rateShape[fi] ? rateShape[fi]
                                    : (sizeof(T) == 4 ? (weno ? 4 : 3) : 2);
    VLSG_CUDA(cudaMemsetAsync(rateCounts + 2, 0, sizeof(unsigned long long), stream));
    {
      Scope sc(this, rateShapeName(shape));
      launchBatchRates(A, weno, shape);
      checkLaunch();
    }
    {
      Scope sc(this, "domain_steps");
      kDomainSteps<<<grid1(nDom), 256, 0, stream>>>(nDom, domRed, domDelta, lfFamily ? 1 : 0, cap,
                                                    out, domUpdates, first ? 1 : 0, errPtr());
      checkLaunch();
    }
    updateRebuild(0.0, out);
    if (!deferMaintain) maintain();
  }

  // CUDA graphs of the batching form's time step.  A batch step reads
  // nothing back until it ends, so its launches can be captured once and
  // replayed.  The host tracks, between steps, which of two mask arrays is
  // current per buffer and which array holds which buffer's visit flags; a
  // captured step is only valid from the host state it was captured in, so
  // graphs are kept per (state, parameters), and a replay leaves the host in
  // the state the captured step ended in.
  struct HostState {
    int cur[MAXB], width[MAXB];
    double bound[MAXB];
    uint8_t live[MAXB], visitOk[MAXB];
    uint8_t *visit[MAXB];
    uint8_t *visitSpare;
  };
  HostState hostState() const {
    HostState h;
    std::memset(&h, 0, sizeof(h));
    for (int b = 0; b < MAXB; ++b) {
      h.cur[b] = buf[b].cur, h.width[b] = buf[b].width, h.bound[b] = buf[b].bound;
      h.live[b] = buf[b].live, h.visitOk[b] = visitOk[b], h.visit[b] = visit[b];
    }
    h.visitSpare = visitSpare;
    return h;
  }
  void setHostState(const HostState &h) {
    for (int b = 0; b < MAXB; ++b) {
      buf[b].cur = h.cur[b], buf[b].width = h.width[b], buf[b].bound = h.bound[b];
      buf[b].live = h.live[b], visitOk[b] = h.visitOk[b], visit[b] = h.visit[b];
    }
    visitSpare = h.visitSpare;
  }
  struct StepGraph {
    HostState pre, post;
    vlsg_advect_params P;
    cudaGraphExec_t exec = nullptr;
    uint64_t launches = 0;
    uint32_t stages = 0;
  };
  std::vector<StepGraph> stepGraphs;
  uint64_t batchSteps = 0;
  void dropGraphs() {
    for (auto &g2 : stepGraphs)
      if (g2.exec) cudaGraphExecDestroy(g2.exec);
    stepGraphs.clear();
  }

  // The device work of one batch step (no host reads).
  void batchStepDevice(const vlsg_advect_params &P) {
    double *dA = domDt, *dB = domDt + nDom, *dC = domDt + 2 * nDom, *tm = domDt + 3 * nDom;
    VLSG_CUDA(cudaMemsetAsync(domUpdates, 0, nDom * sizeof(unsigned long long), stream));
    switch (P.temporal_scheme) {
    case VLSG_RUNGE_KUTTA_2ND_ORDER:
      deferMaintain = P.time_step_ratio <= 0.5;
      saveTop(P, 2);
      stageBatch(P, nullptr, dA, true);
      stageBatch(P, dA, dB, false);
      combineLevelSets(P, 0.5, 0.5);
      endStep();
      break;
    case VLSG_RUNGE_KUTTA_3RD_ORDER:
      deferMaintain = P.time_step_ratio <= 0.5;
      saveTop(P, 3);
      stageBatch(P, nullptr, dA, true);
      stageBatch(P, dA, dB, false);
      combineLevelSets(P, 0.75, 0.25);
      stageBatch(P, dA, dC, false);
      combineLevelSets(P, 1.0 / 3.0, 2.0 / 3.0);
      endStep();
      break;
    default:
      stageBatch(P, nullptr, dA, true);
      break;
    }
    {
      Scope sc(this, "domain_time");
      kDomainTime<<<grid1(nDom), 256, 0, stream>>>(nDom, P.temporal_scheme, dA, dB, dC, tm);
      checkLaunch();
    }
  }

  void applyBatch(const vlsg_advect_params &P, vlsg_advect_result *res) override {
    if (!nDom) throw CudaError("no batch of domains set", VLSG_ERR_STATE);
    const int s = P.spatial_scheme;
    if (schemeWidth(s) < 0) throw CudaError("Advect: Discretization scheme not found.", VLSG_ERR_ARGUMENT);
    if (s == VLSG_LAX_FRIEDRICHS_1ST_ORDER || s == VLSG_LAX_FRIEDRICHS_2ND_ORDER ||
        s == VLSG_STENCIL_LOCAL_LAX_FRIEDRICHS_1ST_ORDER)
      throw CudaError("batching form: global Lax-Friedrichs and Stencil-LLF schemes are not "
                      "supported", VLSG_ERR_ARGUMENT);
    if (P.advection_time != 0.)
      throw CudaError("batching form: one time step per call (advection_time 0)", VLSG_ERR_ARGUMENT);
    if (P.ignore_voids || P.track_point_data || P.save_advection_velocities || P.fp32_compensation)
      throw CudaError("batching form: voids, point data and FP32 compensation are not supported",
                      VLSG_ERR_ARGUMENT);
    if (velCb || updCb) throw CudaError("batching form: device velocity functors only", VLSG_ERR_STATE);
    ++generation;
    deferMaintain = false;
    saveTopAt = 0;
    pdTrack = pdSave = pdHas = false;
    compActive = false;
    loValid = false;
    pristine = false;
    rebuildCutoff = 1.0;
    rebuildWidth = 2;
    pointUpdates = 0;
    stages = 0;
    const uint64_t l0 = launches;
    // rate storage for every active point of the step: at most twice the
    // band the step starts from (sized here, before any capture)
    ensureRateCap((size_t)(2 * defined(L - 1) + 65536));
    double *dA = domDt, *dB = domDt + nDom, *dC = domDt + 2 * nDom, *tm = domDt + 3 * nDom;
    const double *last = P.temporal_scheme == VLSG_RUNGE_KUTTA_2ND_ORDER   ? dB
                         : P.temporal_scheme == VLSG_RUNGE_KUTTA_3RD_ORDER ? dC
                                                                            : dA;
    // the first step runs as it is (it sizes what the step allocates); later
    // steps replay the graph captured from the same host state and
    // parameters, capturing it the first time (not while profiling, whose
    // per-launch events read the device back)
    const HostState pre = hostState();
    StepGraph *hit = nullptr;
    for (auto &sg : stepGraphs)
      if (!std::memcmp(&sg.pre, &pre, sizeof(pre)) && !std::memcmp(&sg.P, &P, sizeof(P))) hit = &sg;
    if (hit) {
      VLSG_CUDA(cudaGraphLaunch(hit->exec, stream));
      setHostState(hit->post);
      launches += hit->launches;
      stages = hit->stages;
    } else if (batchSteps > 0 && !profiling) {
      StepGraph sg;
      sg.pre = pre;
      sg.P = P;
      VLSG_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeRelaxed));
      capturing = true;
      try {
        batchStepDevice(P);
      } catch (...) {
        capturing = false;
        cudaGraph_t gr = nullptr;
        cudaStreamEndCapture(stream, &gr);
        if (gr) cudaGraphDestroy(gr);
        throw;
      }
      capturing = false;
      cudaGraph_t gr = nullptr;
      VLSG_CUDA(cudaStreamEndCapture(stream, &gr));
      const cudaError_t e = cudaGraphInstantiate(&sg.exec, gr, 0);
      cudaGraphDestroy(gr);
      VLSG_CUDA(e);
      sg.post = hostState();
      sg.launches = launches - l0;
      sg.stages = stages;
      VLSG_CUDA(cudaGraphLaunch(sg.exec, stream));
      stepGraphs.push_back(sg);
    } else {
      batchStepDevice(P);
    }
    ++batchSteps;
    std::vector<double> hTime(nDom), hLast(nDom);
    std::vector<unsigned long long> hUpd(nDom);
    VLSG_CUDA(cudaMemcpyAsync(hTime.data(), tm, nDom * sizeof(double), cudaMemcpyDeviceToHost, stream));
    VLSG_CUDA(cudaMemcpyAsync(hLast.data(), last, nDom * sizeof(double), cudaMemcpyDeviceToHost, stream));
    VLSG_CUDA(cudaMemcpyAsync(hUpd.data(), domUpdates, nDom * sizeof(unsigned long long),
                              cudaMemcpyDeviceToHost, stream));
    syncErr("batch advect");
    const uint64_t nl = launches - l0;
    for (int d = 0; d < nDom; ++d) {
      res[d].advected_time = hTime[d];
      res[d].current_time_step = hLast[d];
      res[d].number_of_time_steps = 1;
      res[d].number_of_stages = stages;
      res[d].point_updates = hUpd[d];
      res[d].kernel_launches = nl;
      pointUpdates += hUpd[d];
    }
  }

  // ------------------------------------------------------------ download
  int64_t countDefined(int b) override { return defined(b); }
  int width(int b) const override { return buf[b].width; }

  void queryValues(int b, int64_t n, const int32_t *idx, double *out) override {
    if (n <= 0) return;
    int *di = nullptr;
    double *dv = nullptr;
    VLSG_CUDA(cudaMalloc(&di, n * 3 * sizeof(int)));
    VLSG_CUDA(cudaMalloc(&dv, n * sizeof(double)));
    VLSG_CUDA(cudaMemcpyAsync(di, idx, n * 3 * sizeof(int), cudaMemcpyHostToDevice, stream));
    {
      Scope sc(this, "query");
      kQueryValues<T><<<grid1(n), 256, 0, stream>>>(g, mapView(), view(b), (int)n, di, dv,
                                                     loRead(b));
      checkLaunch();
    }
    VLSG_CUDA(cudaMemcpyAsync(out, dv, n * sizeof(double), cudaMemcpyDeviceToHost, stream));
    VLSG_CUDA(cudaStreamSynchronize(stream));
    cudaFree(di);
    cudaFree(dv);
  }

  // ------------------------------------------------------------ exchange
  template <class V> V *pinned(int k, size_t n) {
    const size_t bytes = std::max<size_t>(n, 1) * sizeof(V);
    if (hs[k].bytes < bytes) {
      if (hs[k].p) VLSG_CUDA(cudaFreeHost(hs[k].p));
      hs[k].p = nullptr;
      hs[k].bytes = 0;
      const size_t grown = bytes + bytes / 4;
      VLSG_CUDA(cudaHostAlloc(&hs[k].p, grown, cudaHostAllocDefault));
      hs[k].bytes = grown;
    }
    return (V *)hs[k].p;
  }
  template <class V> V *scratch(int k, size_t n) {
    const size_t bytes = std::max<size_t>(n, 1) * sizeof(V);
    if (xs[k].bytes < bytes) {
      if (xs[k].p) VLSG_CUDA(cudaFree(xs[k].p));
      xs[k].p = nullptr;
      xs[k].bytes = 0;
      const size_t grown = bytes + bytes / 4;
      VLSG_CUDA(cudaMalloc(&xs[k].p, grown));
      xs[k].bytes = grown;
    }
    return (V *)xs[k].p;
  }
  // Exclusive scan of n counts; the total lands in sums[(n + tile - 1) / tile].
  // Up to SCAN_TOP_THREADS * SCAN_TOP_ITEMS tiles the tile sums are scanned
  // by one block; beyond that (a batch of many domains has a large brick
  // box) they are scanned by this same three-kernel scan, one level deeper.
  void scanExclusive(const uint32_t *in, uint32_t *out, size_t n, uint32_t *sums, int depth = 0) {
    const size_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (nb == 0) {
      VLSG_CUDA(cudaMemsetAsync(sums, 0, sizeof(uint32_t), stream));
      return;
    }
    kScanReduce<<<(unsigned)nb, SCAN_THREADS, 0, stream>>>(in, n, sums);
    if (nb <= (size_t)SCAN_TOP_THREADS * SCAN_TOP_ITEMS) {
      kScanTop<<<1, SCAN_TOP_THREADS, 0, stream>>>(sums, (int)nb);
    } else {
      if (depth >= 1) throw CudaError("exchange: too many elements for the scan", VLSG_ERR_CAPACITY);
      uint32_t *sums2 = scratch<uint32_t>(X_SCAN2, scanScratch(nb) + 64);
      scanExclusive(sums, sums, nb, sums2, depth + 1); // in place: each tile is read before written
      VLSG_CUDA(cudaMemcpyAsync(sums + nb, sums2 + (nb + SCAN_TILE - 1) / SCAN_TILE, sizeof(uint32_t),
                                cudaMemcpyDeviceToDevice, stream));
    }
    kScanApply<<<(unsigned)nb, SCAN_THREADS, 0, stream>>>(in, n, sums, out);
    checkLaunch();
  }
  uint32_t scanTotal(const uint32_t *sums, size_t n) {
    const size_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
    VLSG_CUDA(cudaMemcpyAsync(pinCounters + 30, sums + nb, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                              stream));
    VLSG_CUDA(cudaStreamSynchronize(stream));
    return (uint32_t)pinCounters[30];
  }

  // Points (HRLE order) and runs of buffer b on the device, in the scratch
  // arrays X_IDX / X_VAL / X_OSTART / X_OSIGN.
  // First half of the exchange layout of buffer b: ordered bricks, their
  // rows and slabs, and the points before every segment (P); returns the
  // number of points.  Also the points' bounding box (X_BOX).
  uint32_t pointLayout(int b, int nAlloc) {
    uint32_t *flags = scratch<uint32_t>(X_FLAGS, nBricks);
    uint32_t *pos = scratch<uint32_t>(X_POS, nBricks);
    uint32_t *sums = scratch<uint32_t>(X_SUMS, scanScratch((size_t)std::max(nBricks, nAlloc * 64)) + 64);
    kAllocFlags<<<grid1(nBricks), 256, 0, stream>>>(brickMap, nBricks, flags);
    scanExclusive(flags, pos, nBricks, sums);
    int *ob = scratch<int>(X_OB, nAlloc);
    kOrderedBricks<<<grid1(nBricks), 256, 0, stream>>>(brickMap, nBricks, pos, ob);
    int4 *bounds = scratch<int4>(X_BOUNDS, nAlloc);
    kBrickBounds<<<grid1(nAlloc), 256, 0, stream>>>(g, ob, nAlloc, bounds);
    const size_t nSeg = (size_t)nAlloc * 64;
    uint32_t *C = scratch<uint32_t>(X_C, nSeg);
    uint32_t *P = scratch<uint32_t>(X_P, nSeg);
    int *box = scratch<int>(X_BOX, 8);
    const int boxInit[6] = {INT_MAX, INT_MAX, INT_MAX, INT_MIN, INT_MIN, INT_MIN};
    std::memcpy(pinCounters + 16, boxInit, sizeof(boxInit));
    VLSG_CUDA(cudaMemcpyAsync(box, pinCounters + 16, sizeof(boxInit), cudaMemcpyHostToDevice, stream));
    const uint64_t *def = buf[b].def[buf[b].cur];
    kSegCounts<<<grid1(nSeg), 256, 0, stream>>>(g, ob, nAlloc, brickMap, bounds, def, C, box);
    scanExclusive(C, P, nSeg, sums);
    return scanTotal(sums, nSeg);
  }

  void buildExchange(int b) {
    if (xBuf == b && xGen == generation) return;
    Scope sc(this, "exchange");
    const int nAlloc = readI32(nSlotsPtr());
    const uint32_t nPts = pointLayout(b, nAlloc);
    const size_t nSeg = (size_t)nAlloc * 64;
    int4 *bounds = (int4 *)xs[X_BOUNDS].p;
    uint32_t *P = (uint32_t *)xs[X_P].p;
    uint32_t *sums = (uint32_t *)xs[X_SUMS].p;
    int *box = (int *)xs[X_BOX].p;
    int *ob = (int *)xs[X_OB].p;
    const uint64_t *def = buf[b].def[buf[b].cur];
    int hbox[6];
    VLSG_CUDA(cudaMemcpyAsync(pinCounters + 16, box, sizeof(hbox), cudaMemcpyDeviceToHost, stream));
    VLSG_CUDA(cudaStreamSynchronize(stream));
    std::memcpy(hbox, pinCounters + 16, sizeof(hbox));
    checkLaunch();
    RunBox rb{};
    for (int d = 0; d < 3; ++d) {
      rb.lo[d] = nPts ? hbox[d] - 1 : 0;
      rb.hi[d] = nPts ? hbox[3 + d] + 1 : 0;
    }
    // D = 2: the plane z = 0 alone, without the runs before and after it
    // (the first and last of the list, left out of the merge below)
    if (g.planar) rb.lo[2] = rb.hi[2] = 0;
    rb.ny = rb.hi[1] - rb.lo[1] + 1;
    rb.nz = rb.hi[2] - rb.lo[2] + 1;
    const size_t rows = (size_t)rb.ny * rb.nz;
    int32_t *idx = scratch<int32_t>(X_IDX, 3 * (size_t)nPts);
    double *val = scratch<double>(X_VAL, nPts);
    uint32_t *GC = scratch<uint32_t>(X_GC, nSeg);
    uint32_t *GE = scratch<uint32_t>(X_GE, nSeg);
    uint32_t *rowC = scratch<uint32_t>(X_ROWC, rows);
    uint32_t *rowG = scratch<uint32_t>(X_ROWG, rows);
    uint32_t *PB = scratch<uint32_t>(X_PB, rows);
    uint32_t *GB = scratch<uint32_t>(X_GB, rows);
    uint32_t *sums2 = scratch<uint32_t>(X_KPOS, scanScratch(rows) + 64);
    VLSG_CUDA(cudaMemsetAsync(rowC, 0, rows * sizeof(uint32_t), stream));
    VLSG_CUDA(cudaMemsetAsync(rowG, 0, rows * sizeof(uint32_t), stream));
    kSegScatter<T><<<grid1(nSeg), 256, 0, stream>>>(g, ob, nAlloc, brickMap, nbr, bounds, def,
                                                    buf[b].vals, P, rb, idx, val, GC, rowC, rowG,
                                                    loRead(b));
    scanExclusive(GC, GE, nSeg, sums);
    scanExclusive(rowC, PB, rows, sums2);
    scanExclusive(rowG, GB, rows, sums2);
    const uint32_t gaps = scanTotal(sums2, rows);
    const size_t nRuns = 2 + 2 * (size_t)rb.nz + rows + gaps;
    if (nRuns >= (size_t)UINT32_MAX || (size_t)nPts >= (size_t)INT32_MAX)
      throw CudaError("exchange: level set too large", VLSG_ERR_CAPACITY);
    RunSink<T> sink{scratch<int32_t>(X_RSTART, 3 * nRuns), scratch<int8_t>(X_RSIGN, nRuns),
                    scratch<uint32_t>(X_RPB, nRuns), g, mapView(), view(b)};
    kRunsRows<T><<<grid1(rows), 256, 0, stream>>>(rb, rowC, rowG, PB, GB, idx, nPts,
                                                  (uint32_t)nRuns, sink);
    kRunsGaps<T><<<grid1(nSeg), 256, 0, stream>>>(g, ob, nAlloc, brickMap, nbr, bounds, def, P, GE,
                                                  rb, sink);
    uint32_t *keep = scratch<uint32_t>(X_KEEP, nRuns);
    uint32_t *kpos = scratch<uint32_t>(X_POS, std::max<size_t>(nRuns, nBricks));
    uint32_t *sums3 = scratch<uint32_t>(X_SUMS, scanScratch(std::max<size_t>(nRuns, std::max(nBricks, nAlloc * 64))) + 64);
    const size_t r0 = g.planar ? 1 : 0, nMerge = nRuns - 2 * r0;
    kRunKeep<<<grid1(nMerge), 256, 0, stream>>>(sink.sign + r0, sink.pb + r0, (uint32_t)nMerge,
                                                keep);
    scanExclusive(keep, kpos, nMerge, sums3);
    const uint32_t kept = scanTotal(sums3, nMerge);
    kRunCompact<<<grid1(nMerge), 256, 0, stream>>>(sink.start + 3 * r0, sink.sign + r0, keep, kpos,
                                                   (uint32_t)nMerge,
                                                   scratch<int32_t>(X_OSTART, 3 * (size_t)kept),
                                                   scratch<int8_t>(X_OSIGN, kept));
    checkLaunch();
    syncErr("exchange");
    xBuf = b;
    xGen = generation;
    xPoints = nPts;
    xRuns = kept;
  }

  // Defined points of buffer b in HRLE order; returns their number.
  int64_t compact(int b, int32_t *idxOut, double *valOut, int64_t capOut) override {
    buildExchange(b);
    if (!idxOut || !valOut || xPoints > capOut) return xPoints;
    if (xPoints) {
      VLSG_CUDA(cudaMemcpyAsync(idxOut, xs[X_IDX].p, 3 * sizeof(int32_t) * xPoints,
                                cudaMemcpyDeviceToHost, stream));
      VLSG_CUDA(cudaMemcpyAsync(valOut, xs[X_VAL].p, sizeof(double) * xPoints,
                                cudaMemcpyDeviceToHost, stream));
      VLSG_CUDA(cudaStreamSynchronize(stream));
    }
    return xPoints;
  }
  // Undefined runs of buffer b (HRLE order); returns their number.
  int64_t runs(int b, int32_t *startOut, int8_t *signOut, int64_t capOut) override {
    buildExchange(b);
    if (!startOut || !signOut || xRuns > capOut) return xRuns;
    if (xRuns) {
      VLSG_CUDA(cudaMemcpyAsync(startOut, xs[X_OSTART].p, 3 * sizeof(int32_t) * xRuns,
                                cudaMemcpyDeviceToHost, stream));
      VLSG_CUDA(cudaMemcpyAsync(signOut, xs[X_OSIGN].p, xRuns, cudaMemcpyDeviceToHost, stream));
      VLSG_CUDA(cudaStreamSynchronize(stream));
    }
    return xRuns;
  }

  // ------------------------------------------------------ interface extras
  void queryStaged(int b, int64_t n, const int32_t *idx, double *out, int32_t *di,
                   double *dv) override {
    VLSG_CUDA(cudaMemcpyAsync(di, idx, n * 3 * sizeof(int32_t), cudaMemcpyHostToDevice, stream));
    {
      Scope sc(this, "query");
      kQueryValues<T><<<grid1(n), 256, 0, stream>>>(g, mapView(), view(b), (int)n, di, dv,
                                                     loRead(b));
      checkLaunch();
    }
    VLSG_CUDA(cudaMemcpyAsync(out, dv, n * sizeof(double), cudaMemcpyDeviceToHost, stream));
    VLSG_CUDA(cudaStreamSynchronize(stream));
  }
  void exchange(int b, const int32_t **idx, const double **val, int64_t *n) override {
    buildExchange(b);
    *idx = (const int32_t *)xs[X_IDX].p;
    *val = (const double *)xs[X_VAL].p;
    *n = xPoints;
  }
  void prepareStencilLLF(const std::vector<bool> &isDepo) override { prepareStencil(isDepo); }
  void finalizeStencilLLF() override { finalizeStencil(); }
  // Advect::prepareLS (lsAdvect.hpp:972-1015): Expand to the scheme's width
  void prepareLS(int s) override {
    const int w = schemeWidth(s);
    if (w < 0) throw CudaError("Advect: Discretization scheme not found.", VLSG_ERR_ARGUMENT);
    ++generation; // the exchange format is rebuilt on the next download
    saveTopAt = 0;
    loValid = false;
    pristine = false;
    expand(L - 1, w);
    syncErr("prepareLS");
  }

  uint64_t insideCells(int b) override {
    VLSG_CUDA(cudaMemsetAsync(small + 15, 0, sizeof(unsigned long long), stream));
    kInsideCells<T><<<blocksPass, 256, 0, stream>>>(g, mapView(), view(b), nBricks, small + 15,
                                                    loRead(b));
    checkLaunch();
    return readU64(small + 15);
  }
  int64_t pointData(int b, int64_t *src, double *vel, double *diss, int64_t cap) override {
    if (b != L - 1 || !pdHas) return -1;
    buildExchange(b);
    if (!src || !vel || !diss || xPoints > cap) return xPoints;
    if (!xPoints) return 0;
    const int nAlloc = readI32(nSlotsPtr());
    int64_t *ds = scratch<int64_t>(X_PSRC, xPoints);
    double *dv = scratch<double>(X_PVEL, xPoints);
    double *dd = scratch<double>(X_PDISS, xPoints);
    {
      Scope sc(this, "point_data");
      kSegPointData<T><<<grid1((size_t)nAlloc * 64), 256, 0, stream>>>(
          (const int *)xs[X_OB].p, nAlloc, brickMap, (const int4 *)xs[X_BOUNDS].p,
          buf[b].def[buf[b].cur], (const uint32_t *)xs[X_P].p, pdCells, ds, dv, dd);
      checkLaunch();
    }
    VLSG_CUDA(cudaMemcpyAsync(src, ds, xPoints * sizeof(int64_t), cudaMemcpyDeviceToHost, stream));
    VLSG_CUDA(cudaMemcpyAsync(vel, dv, xPoints * sizeof(double), cudaMemcpyDeviceToHost, stream));
    VLSG_CUDA(cudaMemcpyAsync(diss, dd, xPoints * sizeof(double), cudaMemcpyDeviceToHost, stream));
    VLSG_CUDA(cudaStreamSynchronize(stream));
    return xPoints;
  }
  int64_t surfaceNodes(int b, double **nodes, uint64_t **keys) override {
    buildExchange(b);
    const int64_t n = xPoints;
    const int32_t *idx = (const int32_t *)xs[X_IDX].p;
    const double *val = (const double *)xs[X_VAL].p;
    uint32_t *cnt = nullptr, *off = nullptr, *sums = nullptr;
    VLSG_CUDA(cudaMalloc(&cnt, std::max<int64_t>(n, 1) * sizeof(uint32_t)));
    VLSG_CUDA(cudaMalloc(&off, std::max<int64_t>(n, 1) * sizeof(uint32_t)));
    VLSG_CUDA(cudaMalloc(&sums, (scanScratch(n) + 64) * sizeof(uint32_t)));
    kSurfaceNodes<T><<<grid1(n), 256, 0, stream>>>(g, mapView(), view(b), idx, val, n, cnt, nullptr,
                                                   nullptr, nullptr, loRead(b));
    scanExclusive(cnt, off, n, sums);
    const int64_t m = scanTotal(sums, n);
    VLSG_CUDA(cudaMalloc(nodes, std::max<int64_t>(m, 1) * 3 * sizeof(double)));
    VLSG_CUDA(cudaMalloc(keys, std::max<int64_t>(m, 1) * sizeof(uint64_t)));
    kSurfaceNodes<T><<<grid1(n), 256, 0, stream>>>(g, mapView(), view(b), idx, val, n, cnt, off,
                                                   *nodes, *keys, loRead(b));
    checkLaunch();
    VLSG_CUDA(cudaStreamSynchronize(stream));
    cudaFree(cnt);
    cudaFree(off);
    cudaFree(sums);
    return m;
  }
};

} // namespace
} // namespace vlsg
