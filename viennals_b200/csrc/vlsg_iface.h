// vlsg_iface.h -- host-side types shared by the C ABI unit and the engine
// units (one per storage type, compiled separately so that the FP32 engine
// may use fused multiply-add while the FP64 engine keeps the reference's
// rounding), and the abstract engine the C ABI drives.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "vlsg_common.cuh"

namespace vlsg {

struct CudaError : std::runtime_error {
  int code;
  CudaError(const std::string &m, int c) : std::runtime_error(m), code(c) {}
};

#define VLSG_CUDA(x)                                                           \
  do {                                                                         \
    cudaError_t e_ = (x);                                                      \
    if (e_ != cudaSuccess)                                                     \
      throw vlsg::CudaError(std::string(#x) + ": " + cudaGetErrorString(e_),   \
                            VLSG_ERR_CUDA);                                    \
  } while (0)

// Device array that only grows (contents are not kept when it does).
template <class V> void growDevice(V *&p, size_t &capacity, size_t n) {
  if (p && n <= capacity) return;
  if (p) VLSG_CUDA(cudaFree(p));
  p = nullptr;
  capacity = 0;
  const size_t c = std::max<size_t>(n + n / 4, 16);
  VLSG_CUDA(cudaMalloc(&p, c * sizeof(V)));
  capacity = c;
}

// One uploaded level set, staged on the device until the context builds.
struct StagedLS {
  int32_t *idx = nullptr;      // 3 per point (as given)
  double *vals = nullptr;
  int32_t *runStart = nullptr; // 3 per run
  int8_t *runSign = nullptr;
  size_t capIdx = 0, capVals = 0, capRunStart = 0, capRunSign = 0;
  int64_t n = 0, nRuns = 0;
  int width = 1;
  StagedLS() = default;
  StagedLS(const StagedLS &) = delete;
  StagedLS &operator=(const StagedLS &) = delete;
  StagedLS(StagedLS &&o) noexcept { *this = std::move(o); }
  StagedLS &operator=(StagedLS &&o) noexcept {
    if (this == &o) return *this;
    release();
    idx = o.idx, vals = o.vals, runStart = o.runStart, runSign = o.runSign;
    capIdx = o.capIdx, capVals = o.capVals, capRunStart = o.capRunStart, capRunSign = o.capRunSign;
    n = o.n, nRuns = o.nRuns, width = o.width;
    o.idx = nullptr, o.vals = nullptr, o.runStart = nullptr, o.runSign = nullptr;
    o.capIdx = o.capVals = o.capRunStart = o.capRunSign = 0;
    return *this;
  }
  ~StagedLS() { release(); }
  void release() {
    if (idx) cudaFree(idx);
    if (vals) cudaFree(vals);
    if (runStart) cudaFree(runStart);
    if (runSign) cudaFree(runSign);
    idx = nullptr, vals = nullptr, runStart = nullptr, runSign = nullptr;
    capIdx = capVals = capRunStart = capRunSign = 0;
  }
};

struct KernelTimer {
  std::string name;
  uint64_t launches = 0;
  double ms = 0;
  double bytes = 0;
};

// Expand width of each scheme's prepareLS (lsEngquistOsher.hpp:31,
// lsLaxFriedrichs.hpp:225, lsLocalLocalLaxFriedrichs.hpp:288,
// lsLocalLaxFriedrichs.hpp:55, lsWENO.hpp:44).
inline int schemeWidth(int s) {
  switch (s) {
  case VLSG_ENGQUIST_OSHER_1ST_ORDER: return 3;
  case VLSG_ENGQUIST_OSHER_2ND_ORDER: return 5;
  case VLSG_LAX_FRIEDRICHS_1ST_ORDER: return 3;
  case VLSG_LAX_FRIEDRICHS_2ND_ORDER: return 5;
  case VLSG_LOCAL_LOCAL_LAX_FRIEDRICHS_1ST_ORDER: return 3;
  case VLSG_LOCAL_LOCAL_LAX_FRIEDRICHS_2ND_ORDER: return 5;
  case VLSG_LOCAL_LAX_FRIEDRICHS_1ST_ORDER: return 7;
  case VLSG_LOCAL_LAX_FRIEDRICHS_2ND_ORDER: return 9;
  case VLSG_LOCAL_LAX_FRIEDRICHS_ANALYTICAL_1ST_ORDER: return 7;
  case VLSG_STENCIL_LOCAL_LAX_FRIEDRICHS_1ST_ORDER: return 8;
  case VLSG_WENO_3RD_ORDER: return 5;
  case VLSG_WENO_5TH_ORDER: return 7;
  default: return -1;
  }
}

// One context's device state and the operations the C ABI needs; Engine<T>
// (vlsg_engine.cuh) implements it for T = double and float.
class EngineBase {
public:
  cudaStream_t stream = nullptr;
  vlsg_velocity_desc vel{};
  // host callback mode when set (the functor `vel` is then unused)
  vlsg_velocity_cb velCb = nullptr;
  void *velUser = nullptr;
  vlsg_alpha_cb alphaCb = nullptr; // dissipation alphas with a callback
  void *alphaUser = nullptr;
  vlsg_update_cb updCb = nullptr; // setVelocityUpdateCallback
  void *updUser = nullptr;
  bool profiling = false;
  std::vector<KernelTimer> timers;

  virtual ~EngineBase() = default;
  virtual void build(const GridDev &grid, std::vector<StagedLS> &ls, int margin) = 0;
  virtual void apply(const vlsg_advect_params &P, vlsg_advect_result &r) = 0;
  virtual int64_t countDefined(int b) = 0;
  virtual int width(int b) const = 0;
  // defined points / undefined runs in HRLE order (returns the count; writes
  // only when the capacity suffices)
  virtual int64_t compact(int b, int32_t *idx, double *val, int64_t cap) = 0;
  virtual int64_t runs(int b, int32_t *start, int8_t *sign, int64_t cap) = 0;
  virtual void queryValues(int b, int64_t n, const int32_t *idx, double *out) = 0;
  // the same query through device staging the caller provides
  virtual void queryStaged(int b, int64_t n, const int32_t *idx, double *out, int32_t *dIdx,
                           double *dVal) = 0;
  // comparison support: the exchange arrays of buffer b (device), the
  // inside-cell count, and the zero-crossing nodes (device arrays the caller
  // releases with cudaFree; sorted by cell key)
  virtual void exchange(int b, const int32_t **idx, const double **val, int64_t *n) = 0;
  virtual uint64_t insideCells(int b) = 0;
  // PrepareStencilLocalLaxFriedrichs / FinalizeStencilLocalLaxFriedrichs
  virtual void prepareStencilLLF(const std::vector<bool> &isDepo) = 0;
  virtual void finalizeStencilLLF() = 0;
  virtual void prepareLS(int spatialScheme) = 0;
  virtual int64_t surfaceNodes(int b, double **nodes, uint64_t **keys) = 0;
  // sharding: owned slab (axis -1: all) and the cross-shard reduction
  int ownAxis = -1;
  int64_t ownLo = 0, ownHi = 0;
  vlsg_reduce_cb reduceCb = nullptr;
  void *reduceUser = nullptr;
  // Point data of level set b in download order (source id, saved velocity
  // and dissipation); returns the number of points, or -1 when the level set
  // carries no point data.  Nothing is written when cap is too small.
  virtual int64_t pointData(int b, int64_t *src, double *vel, double *diss, int64_t cap) = 0;
  // batching form: the domain table and one level set holding every domain
  // (stacked in z, in the box `grid` gives), then one time step of all
  // domains with results per domain
  virtual void buildBatch(const GridDev &grid, const std::vector<DomainDev> &doms,
                          const std::vector<int> &domOfBz, const std::vector<double> &delta,
                          const std::vector<vlsg_velocity_desc> &vels,
                          std::vector<StagedLS> &ls) = 0;
  virtual void applyBatch(const vlsg_advect_params &P, vlsg_advect_result *res) = 0;
};

EngineBase *makeEngineF32();
EngineBase *makeEngineF64();

} // namespace vlsg
