// vlsg_api.cu -- the C ABI of libvlsgpu.so (declared in include/vlsg.h).
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <atomic>

#include "vlsg_compare.cuh"
#include "vlsg_iface.h"

using namespace vlsg;

struct vlsg_context {
  int device = 0;
  int precision = VLSG_FP64;
  cudaStream_t stream = nullptr;    // stream in use
  cudaStream_t ownStream = nullptr; // stream created with the context
  std::string err;
  bool hasGrid = false;
  int dim = 3;
  GridDev grid{};
  std::vector<StagedLS> staged;
  bool dirty = true;
  bool hasVel = false;
  vlsg_velocity_desc vel{};
  vlsg_velocity_cb velCb = nullptr; // host callback mode when set
  void *velUser = nullptr;
  vlsg_alpha_cb alphaCb = nullptr;
  void *alphaUser = nullptr;
  vlsg_update_cb updCb = nullptr;
  void *updUser = nullptr;
  vlsg_reduce_cb reduceCb = nullptr; // sharding
  void *reduceUser = nullptr;
  int ownAxis = -1;
  int64_t ownLo = 0, ownHi = 0;
  bool profiling = false;
  std::unique_ptr<EngineBase> eng; // Engine<double> or Engine<float>
  // batching form (vlsg_batch_set_domains): where each domain lies in the
  // shared brick box, and the box's points downloaded once per state
  struct Batch {
    int n = 0;
    std::vector<int64_t> gmin, gmax;        // 3 per domain
    std::vector<int64_t> shift;             // 3 per domain: box index = domain index + shift
    std::vector<int64_t> z0, z1;            // box cell planes [z0, z1) of each domain
    bool cached = false;
    std::vector<int32_t> idx;               // the box's points in HRLE order
    std::vector<double> val;
    std::vector<int64_t> first;             // per domain: first point; [n]: total
    int width = 2;
  };
  std::unique_ptr<Batch> batch;
};

namespace {
std::mutex g_errMutex;
std::string g_lastError;

int fail(vlsg_context *ctx, int code, const std::string &msg) {
  if (ctx) ctx->err = msg;
  std::lock_guard<std::mutex> lk(g_errMutex);
  g_lastError = msg;
  return code;
}

template <class F> int guarded(vlsg_context *ctx, F f) {
  try {
    if (ctx) {
      cudaError_t e = cudaSetDevice(ctx->device);
      if (e != cudaSuccess) return fail(ctx, VLSG_ERR_CUDA, cudaGetErrorString(e));
    }
    return f();
  } catch (const CudaError &e) {
    return fail(ctx, e.code, e.what());
  } catch (const std::exception &e) {
    return fail(ctx, VLSG_ERR_ARGUMENT, e.what());
  }
}

int grid1(size_t n) {
  size_t b = (n + 255) / 256;
  if (b < 1) b = 1;
  if (b > 148 * 32) b = 148 * 32;
  return (int)b;
}

// Staging of vlsg_get_values_noalloc: the query indices (3 x int32 each) of
// at most VLSG_NOALLOC_MAX_QUERIES queries, then their values (double each).
constexpr size_t kNoAllocIdxBytes = (size_t)VLSG_NOALLOC_MAX_QUERIES * 3 * sizeof(int32_t);
constexpr size_t kNoAllocBytes = kNoAllocIdxBytes + (size_t)VLSG_NOALLOC_MAX_QUERIES * sizeof(double);
static_assert(kNoAllocIdxBytes % 256 == 0, "value staging must stay 256-byte aligned");
} // namespace

// The array itself.  In host code this name is only a stand-in for the
// symbol; its device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char vlsg_noalloc_scratch[kNoAllocBytes];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_scratchMutex;
unsigned char *g_scratchAddr[kMaxDevices] = {}; // device address per device

// Device address of the staging array on `device` (the current device);
// looked up on the first call per device.
int noallocScratch(vlsg_context *ctx, int device, unsigned char **out) {
  if (device < 0 || device >= kMaxDevices)
    return fail(ctx, VLSG_ERR_ARGUMENT, "device ordinal out of range for vlsg_get_values_noalloc");
  std::lock_guard<std::mutex> lk(g_scratchMutex);
  if (!g_scratchAddr[device]) {
    unsigned char *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress((void **)&p, vlsg_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(ctx, VLSG_ERR_CUDA,
                  std::string("vlsg_get_values_noalloc: cudaGetSymbolAddress failed: ") +
                      cudaGetErrorString(e));
    g_scratchAddr[device] = p;
  }
  *out = g_scratchAddr[device];
  return VLSG_OK;
}

// Device buffer freed at scope exit (comparison temporaries).
struct TempBuf {
  void *p = nullptr;
  explicit TempBuf(size_t bytes) { VLSG_CUDA(cudaMalloc(&p, bytes ? bytes : 16)); }
  ~TempBuf() { if (p) cudaFree(p); }
  template <class V> V *as() const { return (V *)p; }
};

void compareEngines(EngineBase &ea, int sa, EngineBase &eb, int sb, vlsg_compare_result *r) {
  const int32_t *ia = nullptr, *ib = nullptr;
  const double *va = nullptr, *vb = nullptr;
  int64_t na = 0, nb = 0;
  ea.exchange(sa, &ia, &va, &na);
  eb.exchange(sb, &ib, &vb, &nb);
  cudaStream_t s = ea.stream;
  TempBuf ka(na * sizeof(uint64_t)), kb(nb * sizeof(uint64_t));
  TempBuf acc(2 * sizeof(CompareAcc) + 2 * sizeof(ChamferAcc));
  VLSG_CUDA(cudaMemsetAsync(acc.p, 0, 2 * sizeof(CompareAcc) + 2 * sizeof(ChamferAcc), s));
  CompareAcc *accA = acc.as<CompareAcc>(), *accB = accA + 1;
  ChamferAcc *chA = (ChamferAcc *)(accB + 1), *chB = chA + 1;
  kPointKeys<<<grid1(na), 256, 0, s>>>(ia, na, ka.as<uint64_t>());
  kPointKeys<<<grid1(nb), 256, 0, s>>>(ib, nb, kb.as<uint64_t>());
  kComparePoints<<<grid1(na), 256, 0, s>>>(ka.as<uint64_t>(), va, na, kb.as<uint64_t>(), vb, nb,
                                           1, accA);
  kComparePoints<<<grid1(nb), 256, 0, s>>>(kb.as<uint64_t>(), vb, nb, ka.as<uint64_t>(), va, na,
                                           0, accB);
  VLSG_CUDA(cudaGetLastError());
  VLSG_CUDA(cudaStreamSynchronize(s));
  const uint64_t inA = ea.insideCells(sa), inB = eb.insideCells(sb);
  double *nodesA = nullptr, *nodesB = nullptr;
  uint64_t *keysA = nullptr, *keysB = nullptr;
  const int64_t ma = ea.surfaceNodes(sa, &nodesA, &keysA);
  const int64_t mb = eb.surfaceNodes(sb, &nodesB, &keysB);
  TempBuf hold(16);
  struct Free {
    void *p;
    ~Free() { if (p) cudaFree(p); }
  } f1{nodesA}, f2{nodesB}, f3{keysA}, f4{keysB};
  kNearestNodes<<<grid1(ma), 256, 0, s>>>(nodesA, ma, nodesB, keysB, mb, chA);
  kNearestNodes<<<grid1(mb), 256, 0, s>>>(nodesB, mb, nodesA, keysA, ma, chB);
  VLSG_CUDA(cudaGetLastError());
  CompareAcc h[2];
  ChamferAcc c[2];
  VLSG_CUDA(cudaMemcpyAsync(h, accA, sizeof(h), cudaMemcpyDeviceToHost, s));
  VLSG_CUDA(cudaMemcpyAsync(c, chA, sizeof(c), cudaMemcpyDeviceToHost, s));
  VLSG_CUDA(cudaStreamSynchronize(s));
  std::memset(r, 0, sizeof(*r));
  r->points_a = na, r->points_b = nb;
  r->common_points = (int64_t)h[0].common;
  r->defined_only_a = (int64_t)h[0].onlyDefined, r->defined_only_b = (int64_t)h[1].onlyDefined;
  r->active_a = (int64_t)h[0].active, r->active_b = (int64_t)h[1].active;
  r->active_only_a = (int64_t)h[0].onlyActive, r->active_only_b = (int64_t)h[1].onlyActive;
  std::memcpy(&r->max_abs_diff, &h[0].maxDiff, sizeof(double));
  r->rms_abs_diff = h[0].common ? std::sqrt(h[0].sumSq / (double)h[0].common) : 0.0;
  r->inside_cells_a = (int64_t)inA, r->inside_cells_b = (int64_t)inB;
  r->nodes_a = ma, r->nodes_b = mb;
  const int64_t ra = ma - (int64_t)c[0].unresolved, rb = mb - (int64_t)c[1].unresolved;
  r->chamfer_ab = ra ? c[0].sum / ra : 0.0;
  r->chamfer_ba = rb ? c[1].sum / rb : 0.0;
  r->chamfer_mean = (ra + rb) ? (c[0].sum + c[1].sum) / double(ra + rb) : 0.0;
  r->chamfer_rms = (ra + rb) ? std::sqrt((c[0].sumSq + c[1].sumSq) / double(ra + rb)) : 0.0;
  double mx0, mx1;
  std::memcpy(&mx0, &c[0].maxBits, sizeof(double));
  std::memcpy(&mx1, &c[1].maxBits, sizeof(double));
  r->chamfer_max = std::max(mx0, mx1);
  r->chamfer_unresolved = (int64_t)(c[0].unresolved + c[1].unresolved);
  for (int k = 0; k < 4; ++k) r->diff_above[k] = (int64_t)h[0].above[k];
}

void ensureBuilt(vlsg_context *ctx) {
  if (!ctx->hasGrid) throw CudaError("no grid set (vlsg_set_grid)", VLSG_ERR_STATE);
  if (ctx->staged.empty()) throw CudaError("no level set uploaded", VLSG_ERR_STATE);
  if (!ctx->dirty) return;
  const int margin = 4;
  if (!ctx->eng) {
    // Set-up of vlsg_get_values_noalloc on this device: with lazy module
    // loading (the CUDA default) the static staging array is only placed in
    // device memory when this file's module loads, which the address lookup
    // forces.  Doing it here, while the context sets up and may allocate,
    // keeps the later no-allocation calls from loading the module.
    unsigned char *scratch = nullptr;
    const int rc = noallocScratch(ctx, ctx->device, &scratch);
    if (rc != VLSG_OK) throw CudaError(ctx->err, rc);
    ctx->eng.reset(ctx->precision == VLSG_FP64 ? makeEngineF64() : makeEngineF32());
  }
  ctx->eng->stream = ctx->stream;
  ctx->eng->build(ctx->grid, ctx->staged, margin);
  ctx->dirty = false;
}
} // namespace

extern "C" {

int vlsg_version(void) { return 100; }

const char *vlsg_last_error(const vlsg_context *ctx) {
  if (ctx) return ctx->err.c_str();
  return g_lastError.c_str();
}

void vlsg_default_params(vlsg_advect_params *p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->spatial_scheme = VLSG_ENGQUIST_OSHER_1ST_ORDER;
  p->temporal_scheme = VLSG_FORWARD_EULER;
  p->time_step_ratio = 0.4999;
  p->dissipation_alpha = 1.0;
  p->advection_time = 0.;
  p->calculate_normal_vectors = 1;
  p->adaptive_subdivisions = 20;
  p->check_dissipation = 1;
  p->update_point_data = 1;
}

int vlsg_create(vlsg_context **out, int32_t device, int32_t precision) {
  if (!out) return fail(nullptr, VLSG_ERR_ARGUMENT, "vlsg_create: out is NULL");
  if (precision != VLSG_FP64 && precision != VLSG_FP32)
    return fail(nullptr, VLSG_ERR_ARGUMENT, "vlsg_create: unknown precision");
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || device < 0 || device >= n)
    return fail(nullptr, VLSG_ERR_CUDA,
                std::string("vlsg_create: no CUDA device ") + std::to_string(device) +
                    (e != cudaSuccess ? std::string(": ") + cudaGetErrorString(e) : ""));
  auto *ctx = new vlsg_context();
  ctx->device = device;
  ctx->precision = precision;
  int rc = guarded(ctx, [&] {
    VLSG_CUDA(cudaStreamCreateWithFlags(&ctx->ownStream, cudaStreamNonBlocking));
    ctx->stream = ctx->ownStream;
    return VLSG_OK;
  });
  if (rc != VLSG_OK) {
    delete ctx;
    return rc;
  }
  *out = ctx;
  return VLSG_OK;
}

int vlsg_destroy(vlsg_context *ctx) {
  if (!ctx) return VLSG_OK;
  cudaSetDevice(ctx->device);
  ctx->eng.reset();
  if (ctx->ownStream) cudaStreamDestroy(ctx->ownStream);
  delete ctx;
  return VLSG_OK;
}

int vlsg_set_stream(vlsg_context *ctx, void *stream) {
  if (!ctx) return fail(nullptr, VLSG_ERR_ARGUMENT, "NULL context");
  return guarded(ctx, [&] {
    VLSG_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->stream = stream ? (cudaStream_t)stream : ctx->ownStream;
    if (ctx->eng) ctx->eng->stream = ctx->stream;
    return VLSG_OK;
  });
}

int vlsg_get_stream(vlsg_context *ctx, void **stream) {
  if (!ctx || !stream) return fail(ctx, VLSG_ERR_ARGUMENT, "bad argument");
  *stream = (void *)ctx->stream;
  return VLSG_OK;
}

int vlsg_set_grid(vlsg_context *ctx, int32_t dim, const int64_t *gmin, const int64_t *gmax,
                  const int32_t *bc, double delta) {
  if (!ctx) return fail(nullptr, VLSG_ERR_ARGUMENT, "NULL context");
  if (dim != 2 && dim != 3) return fail(ctx, VLSG_ERR_ARGUMENT, "D must be 2 or 3");
  if (!gmin || !gmax || !bc || !(delta > 0))
    return fail(ctx, VLSG_ERR_ARGUMENT, "vlsg_set_grid: bad argument");
  ctx->batch.reset(); // back to one domain
  GridDev g{};
  // D = 2: the plane z = 0 of a grid periodic in z with period 1 (every z
  // neighbour is the cell itself, every z difference 0)
  if (dim == 2) g.gmin[2] = 0, g.gmax[2] = 1, g.bc[2] = VLSG_PERIODIC_BOUNDARY, g.planar = 1;
  for (int d = 0; d < dim; ++d) {
    if (bc[d] < 0 || bc[d] > 4) return fail(ctx, VLSG_ERR_ARGUMENT, "unknown boundary condition");
    if (gmin[d] < -(1 << 19) || gmax[d] > (1 << 19))
      return fail(ctx, VLSG_ERR_ARGUMENT, "grid index bounds exceed +-2^19");
    g.gmin[d] = (int)gmin[d];
    g.gmax[d] = (int)gmax[d];
    g.bc[d] = bc[d];
    if ((bc[d] == VLSG_PERIODIC_BOUNDARY && gmax[d] - gmin[d] < 1) ||
        (bc[d] == VLSG_REFLECTIVE_BOUNDARY && gmax[d] < gmin[d]))
      return fail(ctx, VLSG_ERR_ARGUMENT, "empty bounded direction");
  }
  g.delta = delta;
  ctx->grid = g;
  ctx->dim = dim;
  ctx->hasGrid = true;
  ctx->dirty = true;
  return VLSG_OK;
}

int vlsg_set_level_set_count(vlsg_context *ctx, int32_t n) {
  if (!ctx) return fail(nullptr, VLSG_ERR_ARGUMENT, "NULL context");
  if (n < 1 || n > VLSG_MAX_LEVEL_SETS)
    return fail(ctx, VLSG_ERR_ARGUMENT, "level set count out of range");
  ctx->staged.resize(n);
  ctx->dirty = true;
  return VLSG_OK;
}

int vlsg_upload_levelset(vlsg_context *ctx, int32_t slot, int64_t n, const int32_t *idx,
                         const double *values, int64_t nRuns, const int32_t *runStart,
                         const int8_t *runSign, int32_t width) {
  if (!ctx) return fail(nullptr, VLSG_ERR_ARGUMENT, "NULL context");
  return guarded(ctx, [&] {
    if (!ctx->hasGrid) return fail(ctx, VLSG_ERR_STATE, "vlsg_set_grid must come first");
    if (slot < 0 || slot >= VLSG_MAX_LEVEL_SETS)
      return fail(ctx, VLSG_ERR_ARGUMENT, "level set slot out of range");
    if (n < 0 || nRuns < 0 || (n > 0 && (!idx || !values)) ||
        (nRuns > 0 && (!runStart || !runSign)))
      return fail(ctx, VLSG_ERR_ARGUMENT, "vlsg_upload_levelset: bad arrays");
    if (n > INT_MAX / 4 || nRuns > INT_MAX / 4)
      return fail(ctx, VLSG_ERR_ARGUMENT, "too many points or runs");
    if ((int)ctx->staged.size() <= slot) ctx->staged.resize(slot + 1);
    // straight to the device; the index mapping, the range check and the run
    // order are handled there when the context builds
    StagedLS &s = ctx->staged[slot];
    growDevice(s.idx, s.capIdx, 3 * (size_t)n);
    growDevice(s.vals, s.capVals, (size_t)n);
    growDevice(s.runStart, s.capRunStart, 3 * (size_t)nRuns);
    growDevice(s.runSign, s.capRunSign, (size_t)nRuns);
    if (n) {
      VLSG_CUDA(cudaMemcpyAsync(s.idx, idx, 3 * n * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream));
      VLSG_CUDA(cudaMemcpyAsync(s.vals, values, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    }
    if (nRuns) {
      VLSG_CUDA(cudaMemcpyAsync(s.runStart, runStart, 3 * nRuns * sizeof(int32_t),
                                cudaMemcpyHostToDevice, ctx->stream));
      VLSG_CUDA(cudaMemcpyAsync(s.runSign, runSign, nRuns, cudaMemcpyHostToDevice, ctx->stream));
    }
    VLSG_CUDA(cudaStreamSynchronize(ctx->stream));
    s.n = n;
    s.nRuns = nRuns;
    s.width = width;
    ctx->dirty = true;
    return VLSG_OK;
  });
}

// ---------------------------------------------------------- batching form
namespace {
constexpr int32_t kInfIndex = (1 << 20) - 2; // run starts below the box: -kInfIndex

// The box's points, downloaded once per state, split by domain.
void batchCache(vlsg_context *ctx) {
  auto &B = *ctx->batch;
  if (B.cached) return;
  const int64_t n = ctx->eng->compact(0, nullptr, nullptr, 0);
  B.idx.resize(3 * (size_t)n);
  B.val.resize((size_t)n);
  ctx->eng->compact(0, B.idx.data(), B.val.data(), n);
  B.width = ctx->eng->width(0);
  // HRLE order is z-major and every domain owns a range of z planes
  B.first.assign(B.n + 1, n);
  int64_t p = 0;
  for (int d = 0; d < B.n; ++d) {
    while (p < n && B.idx[3 * p + 2] < B.z0[d]) ++p;
    B.first[d] = p;
  }
  B.first[B.n] = n;
  B.cached = true;
}

int batchDomain(vlsg_context *ctx, int32_t d) {
  if (!ctx->batch || !ctx->eng) return fail(ctx, VLSG_ERR_STATE, "no batch of domains set");
  if (d < 0 || d >= ctx->batch->n) return fail(ctx, VLSG_ERR_ARGUMENT, "domain out of range");
  return VLSG_OK;
}
} // namespace

int vlsg_batch_set_domains(vlsg_context *ctx, int32_t n, const vlsg_batch_domain *doms) {
  if (!ctx) return fail(nullptr, VLSG_ERR_ARGUMENT, "NULL context");
  if (n <= 0 || !doms) return fail(ctx, VLSG_ERR_ARGUMENT, "vlsg_batch_set_domains: no domains");
  return guarded(ctx, [&] {
    auto B = std::make_unique<vlsg_context::Batch>();
    B->n = n;
    B->gmin.resize(3 * (size_t)n), B->gmax.resize(3 * (size_t)n), B->shift.resize(3 * (size_t)n);
    B->z0.resize(n), B->z1.resize(n);
    std::vector<DomainDev> dd(n);
    std::vector<double> delta(n);
    std::vector<vlsg_velocity_desc> vels(n);
    int64_t nPoints = 0, nRuns = 0, planes = 0, maxBx = 1, maxBy = 1;
    constexpr int margin = 4; // brick planes above and below each band
    for (int32_t d = 0; d < n; ++d) {
      const vlsg_batch_domain &D = doms[d];
      if (!D.grid_min || !D.grid_max || !D.boundary || !D.velocity || D.n_points <= 0 ||
          !D.indices || !D.values || D.n_runs < 0 || (D.n_runs > 0 && (!D.run_start || !D.run_sign)))
        return fail(ctx, VLSG_ERR_ARGUMENT, "vlsg_batch_set_domains: domain " + std::to_string(d) +
                                                ": bad arrays");
      if (D.boundary[0] != VLSG_PERIODIC_BOUNDARY || D.boundary[1] != VLSG_PERIODIC_BOUNDARY ||
          D.boundary[2] != VLSG_INFINITE_BOUNDARY)
        return fail(ctx, VLSG_ERR_ARGUMENT, "batching form: domains must be periodic in x and y "
                                            "and infinite in z");
      for (int k = 0; k < 2; ++k)
        if ((D.grid_max[k] - D.grid_min[k]) % 8 != 0 || D.grid_max[k] <= D.grid_min[k])
          return fail(ctx, VLSG_ERR_ARGUMENT, "batching form: periodic extents must be positive "
                                              "multiples of 8 points");
      int64_t zmin = INT64_MAX, zmax = INT64_MIN;
      for (int64_t i = 0; i < D.n_points; ++i) {
        zmin = std::min<int64_t>(zmin, D.indices[3 * i + 2]);
        zmax = std::max<int64_t>(zmax, D.indices[3 * i + 2]);
      }
      const int64_t zo = (int64_t)std::floor((zmin - 8.0 * margin) / 8.0) * 8;
      const int64_t nbz = (zmax + 8 * margin - zo) / 8 + 1;
      for (int k = 0; k < 3; ++k) B->gmin[3 * d + k] = D.grid_min[k], B->gmax[3 * d + k] = D.grid_max[k];
      B->shift[3 * d + 0] = -D.grid_min[0];
      B->shift[3 * d + 1] = -D.grid_min[1];
      B->shift[3 * d + 2] = 8 * planes - zo;
      B->z0[d] = 8 * planes, B->z1[d] = 8 * (planes + nbz);
      dd[d] = DomainDev{(int)((D.grid_max[0] - D.grid_min[0]) / 8), (int)((D.grid_max[1] - D.grid_min[1]) / 8),
                        (int)planes, (int)(planes + nbz)};
      maxBx = std::max<int64_t>(maxBx, dd[d].nbx), maxBy = std::max<int64_t>(maxBy, dd[d].nby);
      planes += nbz;
      delta[d] = D.grid_delta;
      vels[d] = *D.velocity;
      nPoints += D.n_points, nRuns += D.n_runs;
    }
    if (8 * planes >= (1 << 19) || 8 * maxBx >= (1 << 19) || 8 * maxBy >= (1 << 19) ||
        nPoints > INT_MAX / 4 || nRuns > INT_MAX / 4)
      return fail(ctx, VLSG_ERR_CAPACITY, "batching form: the domains do not fit one brick box");
    // one level set holding every domain, translated into the box
    std::vector<int32_t> idx(3 * (size_t)nPoints), rs(3 * (size_t)nRuns);
    std::vector<double> val((size_t)nPoints);
    std::vector<int8_t> sg((size_t)nRuns);
    std::vector<int> domOfBz((size_t)planes);
    int64_t p = 0, r = 0;
    int width = doms[0].width;
    for (int32_t d = 0; d < n; ++d) {
      const vlsg_batch_domain &D = doms[d];
      const int64_t *sh = &B->shift[3 * (size_t)d];
      width = std::min(width, D.width);
      for (int64_t i = 0; i < D.n_points; ++i, ++p) {
        for (int k = 0; k < 3; ++k) idx[3 * p + k] = (int32_t)(D.indices[3 * i + k] + sh[k]);
        val[p] = D.values[i];
      }
      for (int64_t i = 0; i < D.n_runs; ++i, ++r) {
        const int32_t *q = &D.run_start[3 * i];
        if (q[2] <= -kInfIndex) {
          // before the domain's first point: from the start of its planes
          rs[3 * r] = -kInfIndex, rs[3 * r + 1] = -kInfIndex, rs[3 * r + 2] = (int32_t)B->z0[d];
        } else {
          for (int k = 0; k < 3; ++k)
            rs[3 * r + k] = q[k] <= -kInfIndex ? -kInfIndex : (int32_t)(q[k] + sh[k]);
        }
        sg[r] = D.run_sign[i];
      }
      for (int64_t z = dd[d].bz0; z < dd[d].bz1; ++z) domOfBz[z] = d;
    }
    std::vector<StagedLS> staged(1);
    StagedLS &S = staged[0];
    growDevice(S.idx, S.capIdx, idx.size());
    growDevice(S.vals, S.capVals, val.size());
    growDevice(S.runStart, S.capRunStart, rs.size());
    growDevice(S.runSign, S.capRunSign, sg.size());
    VLSG_CUDA(cudaMemcpyAsync(S.idx, idx.data(), idx.size() * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream));
    VLSG_CUDA(cudaMemcpyAsync(S.vals, val.data(), val.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    if (nRuns) {
      VLSG_CUDA(cudaMemcpyAsync(S.runStart, rs.data(), rs.size() * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream));
      VLSG_CUDA(cudaMemcpyAsync(S.runSign, sg.data(), sg.size(), cudaMemcpyHostToDevice, ctx->stream));
    }
    VLSG_CUDA(cudaStreamSynchronize(ctx->stream));
    S.n = nPoints, S.nRuns = nRuns, S.width = width;
    // the box: every domain from brick (0, 0), its planes stacked in z
    GridDev g{};
    for (int k = 0; k < 3; ++k) g.bc[k] = VLSG_INFINITE_BOUNDARY, g.org[k] = 0;
    g.gmax[0] = (int)(8 * maxBx), g.gmax[1] = (int)(8 * maxBy), g.gmax[2] = (int)(8 * planes);
    g.nb[0] = (int)maxBx, g.nb[1] = (int)maxBy, g.nb[2] = (int)planes;
    g.delta = 1.0; // per domain in the batching form
    if (!ctx->eng) {
      unsigned char *scratch = nullptr;
      const int rc = noallocScratch(ctx, ctx->device, &scratch);
      if (rc != VLSG_OK) throw CudaError(ctx->err, rc);
      ctx->eng.reset(ctx->precision == VLSG_FP64 ? makeEngineF64() : makeEngineF32());
    }
    ctx->eng->stream = ctx->stream;
    ctx->eng->velCb = nullptr, ctx->eng->alphaCb = nullptr, ctx->eng->updCb = nullptr;
    ctx->eng->profiling = ctx->profiling;
    ctx->eng->buildBatch(g, dd, domOfBz, delta, vels, staged);
    ctx->batch = std::move(B);
    ctx->hasGrid = false; // the single-domain entry points need their own grid again
    ctx->staged.clear();
    ctx->dirty = true;
    return VLSG_OK;
  });
}

int vlsg_batch_advect(vlsg_context *ctx, const vlsg_advect_params *params,
                      vlsg_advect_result *results) {
  if (!ctx || !params || !results) return fail(ctx, VLSG_ERR_ARGUMENT, "bad argument");
  return guarded(ctx, [&] {
    if (!ctx->batch || !ctx->eng) return fail(ctx, VLSG_ERR_STATE, "no batch of domains set");
    ctx->eng->stream = ctx->stream;
    ctx->eng->profiling = ctx->profiling;
    ctx->batch->cached = false;
    ctx->eng->applyBatch(*params, results);
    return VLSG_OK;
  });
}

int vlsg_batch_count_points(vlsg_context *ctx, int32_t domain, int64_t *n) {
  if (!ctx || !n) return fail(ctx, VLSG_ERR_ARGUMENT, "bad argument");
  return guarded(ctx, [&] {
    const int rc = batchDomain(ctx, domain);
    if (rc != VLSG_OK) return rc;
    batchCache(ctx);
    *n = ctx->batch->first[domain + 1] - ctx->batch->first[domain];
    return VLSG_OK;
  });
}

int vlsg_batch_download(vlsg_context *ctx, int32_t domain, int64_t capacity, int32_t *idx,
                        double *values, int32_t *width) {
  if (!ctx || capacity < 0) return fail(ctx, VLSG_ERR_ARGUMENT, "bad argument");
  return guarded(ctx, [&] {
    const int rc = batchDomain(ctx, domain);
    if (rc != VLSG_OK) return rc;
    batchCache(ctx);
    auto &B = *ctx->batch;
    const int64_t a = B.first[domain], m = B.first[domain + 1] - a;
    if (width) *width = B.width;
    if (m > capacity) return fail(ctx, VLSG_ERR_CAPACITY, "download capacity too small");
    if (m > 0 && (!idx || !values)) return fail(ctx, VLSG_ERR_ARGUMENT, "bad arrays");
    const int64_t *sh = &B.shift[3 * (size_t)domain];
    for (int64_t i = 0; i < m; ++i) {
      for (int k = 0; k < 3; ++k) idx[3 * i + k] = (int32_t)(B.idx[3 * (a + i) + k] - sh[k]);
      values[i] = B.val[a + i];
    }
    return VLSG_OK;
  });
}

int vlsg_batch_download_runs(vlsg_context *ctx, int32_t domain, int64_t capacity,
                             int32_t *runStart, int8_t *runSign, int64_t *nRuns) {
  if (!ctx || !nRuns || capacity < 0 || (capacity > 0 && (!runStart || !runSign)))
    return fail(ctx, VLSG_ERR_ARGUMENT, "bad argument");
  return guarded(ctx, [&] {
    const int rc = batchDomain(ctx, domain);
    if (rc != VLSG_OK) return rc;
    batchCache(ctx);
    auto &B = *ctx->batch;
    const int64_t a = B.first[domain], m = B.first[domain + 1] - a;
    const int64_t *sh = &B.shift[3 * (size_t)domain];
    // the layout of vlsg_download_runs over the box [min - 1, max + 1] of the
    // domain's points (indices in the domain's own grid)
    int64_t lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    if (m) {
      for (int k = 0; k < 3; ++k) lo[k] = INT64_MAX, hi[k] = INT64_MIN;
      for (int64_t i = 0; i < m; ++i)
        for (int k = 0; k < 3; ++k) {
          const int64_t v = B.idx[3 * (a + i) + k] - sh[k];
          lo[k] = std::min(lo[k], v), hi[k] = std::max(hi[k], v);
        }
      for (int k = 0; k < 3; ++k) --lo[k], ++hi[k];
    }
    const int64_t NI = -kInfIndex;
    auto floorDiv2 = [](int64_t v) { return v >= 0 ? v / 2 : -((-v + 1) / 2); };
    const int64_t cxf = floorDiv2(lo[0] + hi[0]), cyf = floorDiv2(lo[1] + hi[1]);
    struct Ev { int64_t s[3], at[3]; };
    std::vector<Ev> ev;
    auto add = [&](int64_t sx, int64_t sy, int64_t sz, int64_t ax, int64_t ay, int64_t az) {
      ev.push_back(Ev{{sx, sy, sz}, {ax, ay, az}});
    };
    add(NI, NI, NI, cxf, cyf, lo[2] - 1);
    add(NI, NI, hi[2] + 1, cxf, cyf, hi[2] + 1);
    for (int64_t z = lo[2]; z <= hi[2]; ++z) {
      add(NI, NI, z, cxf, lo[1] - 1, z);
      add(NI, hi[1] + 1, z, cxf, hi[1] + 1, z);
    }
    // rows of the box: a run at the head of every row (at its first point, or
    // the whole row), one after every point not followed by its +x neighbour
    const int64_t ny = hi[1] - lo[1] + 1, nz = hi[2] - lo[2] + 1;
    if (ny * nz > ((int64_t)1 << 34)) return fail(ctx, VLSG_ERR_CAPACITY, "runs: box too large");
    std::vector<uint8_t> has((size_t)(ny * nz), 0);
    auto P = [&](int64_t i, int k) { return B.idx[3 * (a + i) + k] - sh[k]; };
    for (int64_t i = 0; i < m; ++i) {
      const int64_t x = P(i, 0), y = P(i, 1), z = P(i, 2);
      const bool first = i == 0 || P(i - 1, 1) != y || P(i - 1, 2) != z;
      const bool last = i + 1 == m || P(i + 1, 1) != y || P(i + 1, 2) != z;
      if (first) {
        has[(size_t)((z - lo[2]) * ny + (y - lo[1]))] = 1;
        add(NI, y, z, x - 1, y, z);
      }
      if (last || P(i + 1, 0) > x + 1) add(x + 1, y, z, x + 1, y, z);
    }
    for (int64_t z = lo[2]; z <= hi[2]; ++z)
      for (int64_t y = lo[1]; y <= hi[1]; ++y)
        if (!has[(size_t)((z - lo[2]) * ny + (y - lo[1]))]) add(NI, y, z, lo[0], y, z);
    // signs of the cells the runs start at, through the domain's query
    const int64_t ne = (int64_t)ev.size();
    std::vector<int32_t> q(3 * (size_t)ne);
    for (int64_t i = 0; i < ne; ++i)
      for (int k = 0; k < 3; ++k) q[3 * i + k] = (int32_t)ev[i].at[k];
    std::vector<double> vals((size_t)ne);
    const int qrc = vlsg_batch_get_values(ctx, domain, ne, q.data(), vals.data());
    if (qrc != VLSG_OK) return qrc;
    auto key = [](const int64_t *c) {
      return ((uint64_t)(c[2] + (1 << 20)) << 42) | ((uint64_t)(c[1] + (1 << 20)) << 21) |
             (uint64_t)(c[0] + (1 << 20));
    };
    std::vector<int64_t> o((size_t)ne);
    for (int64_t i = 0; i < ne; ++i) o[i] = i;
    std::stable_sort(o.begin(), o.end(),
                     [&](int64_t x, int64_t y) { return key(ev[x].s) < key(ev[y].s); });
    std::vector<uint64_t> pk((size_t)m);
    for (int64_t i = 0; i < m; ++i) {
      const int64_t c[3] = {P(i, 0), P(i, 1), P(i, 2)};
      pk[i] = key(c);
    }
    // drop a run that repeats the previous run's sign with no point between
    std::vector<int64_t> keepIdx;
    int8_t prevSign = 0;
    int64_t prevBefore = -1;
    for (int64_t j = 0; j < ne; ++j) {
      const Ev &e = ev[o[j]];
      const int8_t sg = vals[o[j]] < 0 ? -1 : 1;
      const int64_t before = std::lower_bound(pk.begin(), pk.end(), key(e.s)) - pk.begin();
      if (j == 0 || sg != prevSign || before != prevBefore) keepIdx.push_back(o[j]);
      prevSign = sg, prevBefore = before;
      vals[o[j]] = sg;
    }
    *nRuns = (int64_t)keepIdx.size();
    if (capacity < *nRuns) return fail(ctx, VLSG_ERR_CAPACITY, "run capacity too small");
    for (size_t i = 0; i < keepIdx.size(); ++i) {
      for (int k = 0; k < 3; ++k) runStart[3 * i + k] = (int32_t)ev[keepIdx[i]].s[k];
      runSign[i] = (int8_t)vals[keepIdx[i]];
    }
    return VLSG_OK;
  });
}

int vlsg_batch_get_values(vlsg_context *ctx, int32_t domain, int64_t n, const int32_t *idx,
                          double *values) {
  if (!ctx || n < 0 || (n > 0 && (!idx || !values)))
    return fail(ctx, VLSG_ERR_ARGUMENT, "bad argument");
  return guarded(ctx, [&] {
    const int rc = batchDomain(ctx, domain);
    if (rc != VLSG_OK) return rc;
    if (n > INT_MAX / 4) return fail(ctx, VLSG_ERR_ARGUMENT, "too many queries");
    auto &B = *ctx->batch;
    const int64_t *sh = &B.shift[3 * (size_t)domain];
    const int64_t *lo = &B.gmin[3 * (size_t)domain], *hi = &B.gmax[3 * (size_t)domain];
    std::vector<int32_t> q(3 * (size_t)n);
    for (int64_t i = 0; i < n; ++i) {
      for (int k = 0; k < 2; ++k) { // periodic in x and y
        const int64_t e = hi[k] - lo[k];
        int64_t c = (idx[3 * i + k] - lo[k]) % e;
        if (c < 0) c += e;
        q[3 * i + k] = (int32_t)(lo[k] + c + sh[k]);
      }
      // z beyond the domain's planes: its first / last plane (no band there)
      const int64_t z = std::min(std::max<int64_t>(idx[3 * i + 2] + sh[2], B.z0[domain]), B.z1[domain] - 1);
      q[3 * i + 2] = (int32_t)z;
    }
    ctx->eng->queryValues(0, n, q.data(), values);
    return VLSG_OK;
  });
}

int vlsg_count_points(vlsg_context *ctx, int32_t slot, int64_t *n) {
  if (!ctx || !n) return fail(ctx, VLSG_ERR_ARGUMENT, "bad argument");
  return guarded(ctx, [&] {
    ensureBuilt(ctx);
    if (slot < 0 || slot >= (int)ctx->staged.size())
      return fail(ctx, VLSG_ERR_ARGUMENT, "level set slot out of range");
    *n = ctx->eng->countDefined(slot);
    return VLSG_OK;
  });
}

int vlsg_download_levelset(vlsg_context *ctx, int32_t slot, int64_t capacity, int32_t *idx,
                           double *values, int32_t *width) {
  if (!ctx) return fail(nullptr, VLSG_ERR_ARGUMENT, "NULL context");
  return guarded(ctx, [&] {
    ensureBuilt(ctx);
    if (slot < 0 || slot >= (int)ctx->staged.size())
      return fail(ctx, VLSG_ERR_ARGUMENT, "level set slot out of range");
    if (width) *width = ctx->eng->width(slot);
    const int64_t n = ctx->eng->compact(slot, idx, values, capacity);
    if (n > capacity) return fail(ctx, VLSG_ERR_CAPACITY, "download capacity too small");
    return VLSG_OK;
  });
}

int vlsg_download_runs(vlsg_context *ctx, int32_t slot, int64_t capacity, int32_t *runStart,
                       int8_t *runSign, int64_t *nRuns) {
  if (!ctx || !nRuns || capacity < 0 || (capacity > 0 && (!runStart || !runSign)))
    return fail(ctx, VLSG_ERR_ARGUMENT, "bad argument");
  return guarded(ctx, [&] {
    ensureBuilt(ctx);
    if (slot < 0 || slot >= (int)ctx->staged.size())
      return fail(ctx, VLSG_ERR_ARGUMENT, "level set slot out of range");
    const int64_t n = ctx->eng->runs(slot, capacity > 0 ? runStart : nullptr,
                                     capacity > 0 ? runSign : nullptr, capacity);
    *nRuns = n;
    if (n > capacity) return fail(ctx, VLSG_ERR_CAPACITY, "run capacity too small");
    return VLSG_OK;
  });
}

int vlsg_download_point_data(vlsg_context *ctx, int32_t slot, int64_t capacity,
                             int64_t *source, double *velocity, double *dissipation,
                             int32_t *has_point_data) {
  if (!ctx || !has_point_data || capacity < 0 ||
      (capacity > 0 && (!source || !velocity || !dissipation)))
    return fail(ctx, VLSG_ERR_ARGUMENT, "bad argument");
  return guarded(ctx, [&] {
    ensureBuilt(ctx);
    if (slot < 0 || slot >= (int)ctx->staged.size())
      return fail(ctx, VLSG_ERR_ARGUMENT, "level set slot out of range");
    if (slot != (int)ctx->staged.size() - 1)
      return fail(ctx, VLSG_ERR_ARGUMENT, "point data is kept for the top level set only");
    const int64_t n = ctx->eng->pointData(slot, nullptr, nullptr, nullptr, 0);
    *has_point_data = n >= 0 ? 1 : 0;
    if (n < 0) return VLSG_OK;
    if (n > capacity) return fail(ctx, VLSG_ERR_CAPACITY, "point data capacity too small");
    ctx->eng->pointData(slot, source, velocity, dissipation, capacity);
    return VLSG_OK;
  });
}

int vlsg_get_values(vlsg_context *ctx, int32_t slot, int64_t n, const int32_t *idx,
                    double *values) {
  if (!ctx || n < 0 || (n > 0 && (!idx || !values)))
    return fail(ctx, VLSG_ERR_ARGUMENT, "bad argument");
  return guarded(ctx, [&] {
    ensureBuilt(ctx);
    if (slot < 0 || slot >= (int)ctx->staged.size())
      return fail(ctx, VLSG_ERR_ARGUMENT, "level set slot out of range");
    if (n > INT_MAX / 4) return fail(ctx, VLSG_ERR_ARGUMENT, "too many queries");
    ctx->eng->queryValues(slot, n, idx, values);
    return VLSG_OK;
  });
}

// Same queries as vlsg_get_values, staged in the library's static device
// array instead of per-call device buffers: no cudaMalloc, no cudaFree.
int vlsg_get_values_noalloc(vlsg_context *ctx, int32_t slot, int64_t n, const int32_t *idx,
                            double *values) {
  if (!ctx || n < 0 || (n > 0 && (!idx || !values)))
    return fail(ctx, VLSG_ERR_ARGUMENT, "bad argument");
  if (n > VLSG_NOALLOC_MAX_QUERIES)
    return fail(ctx, VLSG_ERR_CAPACITY,
                "vlsg_get_values_noalloc: " + std::to_string(n) + " queries exceed the maximum of " +
                    std::to_string(VLSG_NOALLOC_MAX_QUERIES) + " per call");
  return guarded(ctx, [&] {
    if (!ctx->hasGrid || ctx->staged.empty() || ctx->dirty)
      return fail(ctx, VLSG_ERR_STATE,
                  "vlsg_get_values_noalloc: the level sets are not on the device yet (moving them "
                  "there allocates); call vlsg_count_points or vlsg_advect first");
    if (slot < 0 || slot >= (int)ctx->staged.size())
      return fail(ctx, VLSG_ERR_ARGUMENT, "level set slot out of range");
    unsigned char *scratch = nullptr;
    const int rc = noallocScratch(ctx, ctx->device, &scratch);
    if (rc != VLSG_OK) return rc;
    if (n == 0) return VLSG_OK;
    int32_t *di = (int32_t *)scratch;
    double *dv = (double *)(scratch + kNoAllocIdxBytes);
    ctx->eng->queryStaged(slot, n, idx, values, di, dv);
    return VLSG_OK;
  });
}

int vlsg_compare(vlsg_context *a, int32_t slotA, vlsg_context *b, int32_t slotB,
                 vlsg_compare_result *out) {
  if (!a || !b || !out) return fail(a, VLSG_ERR_ARGUMENT, "bad argument");
  if (a->device != b->device) return fail(a, VLSG_ERR_ARGUMENT, "contexts on different devices");
  return guarded(a, [&] {
    ensureBuilt(a);
    ensureBuilt(b);
    if (slotA < 0 || slotA >= (int)a->staged.size() || slotB < 0 || slotB >= (int)b->staged.size())
      return fail(a, VLSG_ERR_ARGUMENT, "level set slot out of range");
    compareEngines(*a->eng, slotA, *b->eng, slotB, out);
    return VLSG_OK;
  });
}

int vlsg_set_velocity_update_callback(vlsg_context *ctx, vlsg_update_cb cb, void *user) {
  if (!ctx) return fail(nullptr, VLSG_ERR_ARGUMENT, "NULL context");
  ctx->updCb = cb;
  ctx->updUser = cb ? user : nullptr;
  return VLSG_OK;
}

int vlsg_prepare_stencil_llf(vlsg_context *ctx, const int32_t *is_depo, int32_t n) {
  if (!ctx || n < 0 || (n > 0 && !is_depo)) return fail(ctx, VLSG_ERR_ARGUMENT, "bad argument");
  if (ctx->staged.empty()) return fail(ctx, VLSG_ERR_STATE, "no level set uploaded");
  return guarded(ctx, [&] {
    ensureBuilt(ctx);
    std::vector<bool> depo(n);
    for (int32_t i = 0; i < n; ++i) depo[i] = is_depo[i] != 0;
    ctx->eng->prepareStencilLLF(depo);
    return VLSG_OK;
  });
}

int vlsg_finalize_stencil_llf(vlsg_context *ctx) {
  if (!ctx) return fail(ctx, VLSG_ERR_ARGUMENT, "bad argument");
  if (ctx->staged.size() < 2)
    return fail(ctx, VLSG_ERR_STATE, "FinalizeStencilLocalLaxFriedrichs needs two level sets");
  return guarded(ctx, [&] {
    ensureBuilt(ctx);
    ctx->eng->finalizeStencilLLF();
    return VLSG_OK;
  });
}

int vlsg_prepare_ls(vlsg_context *ctx, int32_t spatial_scheme) {
  if (!ctx) return fail(ctx, VLSG_ERR_ARGUMENT, "bad argument");
  if (ctx->staged.empty()) return fail(ctx, VLSG_ERR_STATE, "No level sets passed to Advect.");
  return guarded(ctx, [&] {
    ensureBuilt(ctx);
    ctx->eng->prepareLS(spatial_scheme);
    return VLSG_OK;
  });
}

int vlsg_set_velocity_functor(vlsg_context *ctx, const vlsg_velocity_desc *v) {
  if (!ctx || !v) return fail(ctx, VLSG_ERR_ARGUMENT, "bad argument");
  if (v->n_materials < 1 || v->n_materials > VLSG_MAX_MATERIALS)
    return fail(ctx, VLSG_ERR_ARGUMENT, "n_materials out of range");
  ctx->vel = *v;
  ctx->velCb = nullptr;
  ctx->velUser = nullptr;
  ctx->hasVel = true;
  return VLSG_OK;
}

int vlsg_set_velocity_callback(vlsg_context *ctx, vlsg_velocity_cb cb, void *user) {
  if (!ctx || !cb) return fail(ctx, VLSG_ERR_ARGUMENT, "bad argument");
  ctx->velCb = cb;
  ctx->velUser = user;
  ctx->hasVel = true;
  return VLSG_OK;
}

int vlsg_set_dissipation_alpha_callback(vlsg_context *ctx, vlsg_alpha_cb cb, void *user) {
  if (!ctx) return fail(nullptr, VLSG_ERR_ARGUMENT, "NULL context");
  ctx->alphaCb = cb;
  ctx->alphaUser = cb ? user : nullptr;
  return VLSG_OK;
}

int vlsg_advect(vlsg_context *ctx, const vlsg_advect_params *p, vlsg_advect_result *r) {
  if (!ctx || !p || !r) return fail(ctx, VLSG_ERR_ARGUMENT, "bad argument");
  // Advect::apply validation, lsAdvect.hpp:1019-1027
  if (ctx->staged.empty()) return fail(ctx, VLSG_ERR_STATE, "No level sets passed to Advect. Not advecting.");
  if (!ctx->hasVel)
    return fail(ctx, VLSG_ERR_STATE, "No velocity field passed to Advect. Not advecting.");
  if (schemeWidth(p->spatial_scheme) < 0)
    return fail(ctx, VLSG_ERR_ARGUMENT, "Advect: Discretization scheme not found.");
  if (p->temporal_scheme < 0 || p->temporal_scheme > 2)
    return fail(ctx, VLSG_ERR_ARGUMENT, "unknown temporal scheme");
  if (ctx->ownAxis >= 0 && p->spatial_scheme == VLSG_STENCIL_LOCAL_LAX_FRIEDRICHS_1ST_ORDER)
    return fail(ctx, VLSG_ERR_ARGUMENT,
                "an owned region (sharding) is not supported with STENCIL_LOCAL_LAX_FRIEDRICHS");
  return guarded(ctx, [&] {
    // profiling: the timers of this call include the build of a fresh upload
    const bool hadEngine = ctx->eng != nullptr;
    if (hadEngine) {
      ctx->eng->profiling = ctx->profiling;
      if (ctx->profiling) ctx->eng->timers.clear();
    }
    ensureBuilt(ctx);
    EngineBase &e = *ctx->eng;
    e.vel = ctx->vel;
    e.velCb = ctx->velCb;
    e.velUser = ctx->velUser;
    e.alphaCb = ctx->velCb ? ctx->alphaCb : nullptr;
    e.alphaUser = ctx->alphaUser;
    e.updCb = ctx->updCb;
    e.updUser = ctx->updUser;
    e.reduceCb = ctx->reduceCb;
    e.reduceUser = ctx->reduceUser;
    e.ownAxis = ctx->ownAxis;
    e.ownLo = ctx->ownLo;
    e.ownHi = ctx->ownHi;
    e.profiling = ctx->profiling;
    if (ctx->profiling && !hadEngine) e.timers.clear();
    e.apply(*p, *r);
    return VLSG_OK;
  });
}

int vlsg_set_owned_region(vlsg_context *ctx, int32_t axis, int64_t lo, int64_t hi) {
  if (!ctx) return fail(nullptr, VLSG_ERR_ARGUMENT, "NULL context");
  if (axis != -1 && axis != 2)
    return fail(ctx, VLSG_ERR_ARGUMENT, "vlsg_set_owned_region: axis must be 2 (or -1: all)");
  if (axis == 2 && !(lo < hi)) return fail(ctx, VLSG_ERR_ARGUMENT, "vlsg_set_owned_region: empty");
  if (axis == 2 && ctx->hasGrid && ctx->dim == 2)
    return fail(ctx, VLSG_ERR_ARGUMENT, "vlsg_set_owned_region: D = 2 has no z slabs to own");
  ctx->ownAxis = axis;
  ctx->ownLo = lo;
  ctx->ownHi = hi;
  return VLSG_OK;
}

int vlsg_set_reduction_callback(vlsg_context *ctx, vlsg_reduce_cb cb, void *user) {
  if (!ctx) return fail(nullptr, VLSG_ERR_ARGUMENT, "NULL context");
  ctx->reduceCb = cb;
  ctx->reduceUser = user;
  return VLSG_OK;
}

int vlsg_advect_batch(vlsg_context **ctxs, int32_t n, const vlsg_advect_params *params,
                      vlsg_advect_result *results, int32_t threads) {
  if (!ctxs || !params || !results || n < 0)
    return fail(nullptr, VLSG_ERR_ARGUMENT, "vlsg_advect_batch: bad argument");
  for (int32_t i = 0; i < n; ++i)
    if (!ctxs[i]) return fail(nullptr, VLSG_ERR_ARGUMENT, "vlsg_advect_batch: NULL context");
  const int nt = std::max(1, std::min<int>(threads > 0 ? threads : 32, n));
  std::vector<int> status(n, VLSG_OK);
  std::atomic<int> next{0};
  auto worker = [&] {
    for (int i = next.fetch_add(1); i < n; i = next.fetch_add(1))
      status[i] = vlsg_advect(ctxs[i], params, &results[i]);
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < nt; ++t) pool.emplace_back(worker);
  worker();
  for (auto &th : pool) th.join();
  for (int32_t i = 0; i < n; ++i)
    if (status[i] != VLSG_OK) return status[i];
  return VLSG_OK;
}

int vlsg_set_profiling(vlsg_context *ctx, int32_t on) {
  if (!ctx) return fail(nullptr, VLSG_ERR_ARGUMENT, "NULL context");
  ctx->profiling = on != 0;
  return VLSG_OK;
}

int vlsg_get_kernel_stats(vlsg_context *ctx, int32_t capacity, vlsg_kernel_stat *out,
                          int32_t *count) {
  if (!ctx || !count) return fail(ctx, VLSG_ERR_ARGUMENT, "bad argument");
  auto fill = [&](EngineBase &e) {
    *count = (int32_t)e.timers.size();
    for (int i = 0; i < (int)e.timers.size() && i < capacity && out; ++i) {
      std::memset(&out[i], 0, sizeof(out[i]));
      std::snprintf(out[i].name, sizeof(out[i].name), "%s", e.timers[i].name.c_str());
      out[i].launches = e.timers[i].launches;
      out[i].device_ms = e.timers[i].ms;
      out[i].algorithmic_bytes = e.timers[i].bytes;
    }
    return 0;
  };
  if (ctx->eng) fill(*ctx->eng);
  else *count = 0;
  return VLSG_OK;
}

} // extern "C"
