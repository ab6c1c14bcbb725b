// ladds_gpu.cu -- C ABI of the B200 hot path (see include/ladds_gpu.h).
//
// One context = one device, one stream, the device-resident population in two
// SoA copies (current + alternate; a conjunction scan gathers the current copy
// into cell order in the alternate one and swaps them) plus a third copy used
// to roll a ladds_gpu_step call back when it has to be re-run.
//
// A scan iteration is: ephemeris of the three stage times -> constant memory,
// Yoshida step with the cell key of the end position (one kernel), radix
// sort of (key, index), gather into cell order, row-start table, pair scan.
// Multi-iteration calls are captured once into a CUDA graph per (iterations,
// iteration % k, current buffer) and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/ladds_gpu.h"
#include "conjunction.cuh"
#include "propagate.cuh"
#include "radix_sort.cuh"

using namespace ladds;

namespace {

// c_eph is per device: calls on one device are serialised.
std::mutex g_deviceMutex[64];

__global__ void k_advance(int64_t *iter, int by) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *iter += by;
}
__global__ void k_ephemeris_dev(EphEntry *__restrict__ out, int nSteps, const int64_t *__restrict__ iterPtr,
                                double t0, double dt, double hc1, double hc2, double jdEpoch, double theta0) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 3 * nSteps) return;
  const int st = i / 3, stage = i % 3;
  const double tn = t0 + (double)(*iterPtr + st) * dt;
  double tau = tn + hc1;
  if (stage >= 1) tau += hc2;
  if (stage >= 2) tau += hc2;
  ephemeris(jdEpoch, theta0, tau, out[i]);
}

inline int blocksFor(size_t n, int b) { return (int)((n + (size_t)b - 1) / (size_t)b); }

enum Phase { kPhProp = 0, kPhSort = 1, kPhCell = 2, kPhScan = 3, kPhCount = 4 };

}  // namespace

struct ladds_gpu_ctx {
  ladds_gpu_config cfg{};
  GridDesc grid{};
  PropConsts pc{};
  ScanConsts sc{};
  double theta0 = 0;
  int dev = 0;
  cudaStream_t st = nullptr;
  size_t n = 0, cap = 0;
  DevState cur{}, alt{}, snap{};
  uint32_t *keys0 = nullptr, *keys1 = nullptr, *vals0 = nullptr, *vals1 = nullptr;
  uint32_t *sortedKeys = nullptr, *perm = nullptr;  // results of the last sort
  uint32_t *counts = nullptr, *totals = nullptr;
  uint32_t *rowStart = nullptr;
  uint32_t nRows = 0;
  uint32_t *scratchA = nullptr, *scratchB = nullptr, *scratchC = nullptr, *blockSums = nullptr;
  double4 *pos4 = nullptr;  // packed positions in cell order (pair-scan candidate test)
  ladds_pair *dPairs = nullptr;
  size_t pairCap = 0;
  unsigned long long *dCount = nullptr;
  unsigned *dStatus = nullptr;
  EphEntry *dEph = nullptr;
  int64_t *dIter = nullptr;
  int64_t hostIter = 0;
  bool orderValid = false;
  bool profiling = false;
  std::vector<std::tuple<int, cudaEvent_t, cudaEvent_t>> events;
  std::vector<cudaEvent_t> eventPool;
  ladds_phase_times times{};
  cudaEvent_t callStart = nullptr, callEnd = nullptr;
  std::map<std::tuple<int, int, int, size_t, size_t>, cudaGraphExec_t> graphs;
  std::string err;
  double *homeX = nullptr;  // x array of the buffer that was current at allocation
};

namespace {

int fail(ladds_gpu_ctx *c, int code, const std::string &msg) {
  if (c) c->err = msg;
  return code;
}

#define CK(call)                                                                                    \
  do {                                                                                              \
    cudaError_t e_ = (call);                                                                        \
    if (e_ != cudaSuccess)                                                                          \
      return fail(c, LADDS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));           \
  } while (0)

void freeState(DevState &s) {
  void *ptrs[] = {s.x, s.y, s.z, s.vx, s.vy, s.vz, s.aom, s.bc, s.radius, s.id, s.parent, s.tag};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  s = DevState{};
}

cudaError_t allocState(DevState &s, size_t cap) {
  s = DevState{};
  double **d[] = {&s.x, &s.y, &s.z, &s.vx, &s.vy, &s.vz, &s.aom, &s.bc, &s.radius};
  for (double **p : d) {
    cudaError_t e = cudaMalloc(p, cap * sizeof(double));
    if (e != cudaSuccess) return e;
  }
  cudaError_t e = cudaMalloc(&s.id, cap * sizeof(uint64_t));
  if (e == cudaSuccess) e = cudaMalloc(&s.parent, cap * sizeof(uint64_t));
  if (e == cudaSuccess) e = cudaMalloc(&s.tag, cap * sizeof(uint32_t));
  return e;
}

cudaError_t copyState(const DevState &src, const DevState &dst, size_t n, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  const double *sd[] = {src.x, src.y, src.z, src.vx, src.vy, src.vz, src.aom, src.bc, src.radius};
  double *dd[] = {dst.x, dst.y, dst.z, dst.vx, dst.vy, dst.vz, dst.aom, dst.bc, dst.radius};
  for (int k = 0; k < 9; ++k) {
    cudaError_t e = cudaMemcpyAsync(dd[k], sd[k], n * sizeof(double), cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
  }
  cudaError_t e = cudaMemcpyAsync(dst.id, src.id, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dst.parent, src.parent, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dst.tag, src.tag, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st);
  return e;
}

void dropGraphs(ladds_gpu_ctx *c) {
  for (auto &kv : c->graphs) cudaGraphExecDestroy(kv.second);
  c->graphs.clear();
}

void freeBuffers(ladds_gpu_ctx *c) {
  freeState(c->cur);
  freeState(c->alt);
  freeState(c->snap);
  void *ptrs[] = {c->keys0, c->keys1, c->vals0, c->vals1, c->counts, c->scratchA, c->scratchB, c->scratchC,
                  c->blockSums};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (c->pos4) cudaFree(c->pos4);
  c->pos4 = nullptr;
  c->keys0 = c->keys1 = c->vals0 = c->vals1 = c->counts = nullptr;
  c->scratchA = c->scratchB = c->scratchC = c->blockSums = nullptr;
  c->sortedKeys = c->perm = nullptr;
  c->cap = 0;
}

int ensureCapacity(ladds_gpu_ctx *c, size_t need) {
  if (need <= c->cap) return LADDS_OK;
  if (need > kMaxObjects) return fail(c, LADDS_ERR_INVALID_ARG, "population exceeds 2^28 - 1 objects");
  size_t newCap = std::max<size_t>({need, c->cap + c->cap / 2, 4096});
  newCap = std::min(newCap, kMaxObjects);
  DevState ncur, nalt, nsnap;
  cudaError_t e = allocState(ncur, newCap);
  if (e == cudaSuccess) e = allocState(nalt, newCap);
  if (e == cudaSuccess) e = allocState(nsnap, newCap);
  if (e != cudaSuccess) {
    freeState(ncur);
    freeState(nalt);
    freeState(nsnap);
    cudaGetLastError();
    return fail(c, LADDS_ERR_ALLOC, std::string("device allocation failed: ") + cudaGetErrorString(e));
  }
  if (c->n) {
    e = copyState(c->cur, ncur, c->n, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    if (e != cudaSuccess) return fail(c, LADDS_ERR_CUDA, cudaGetErrorString(e));
  }
  const size_t n = c->n;
  freeBuffers(c);
  c->n = n;
  c->cur = ncur;
  c->alt = nalt;
  c->snap = nsnap;
  c->homeX = ncur.x;
  const size_t maxTiles = (newCap + kSortTile - 1) / kSortTile;
  const size_t scanBlocks = (newCap + 1 + kScanBlock - 1) / kScanBlock;
  uint32_t **u[] = {&c->keys0, &c->keys1, &c->vals0, &c->vals1, &c->scratchA, &c->scratchB, &c->scratchC};
  for (uint32_t **p : u) {
    if (cudaMalloc(p, (newCap + 1) * sizeof(uint32_t)) != cudaSuccess) {
      cudaGetLastError();
      return fail(c, LADDS_ERR_ALLOC, "device allocation failed (sort buffers)");
    }
  }
  if (cudaMalloc(&c->counts, (size_t)kRadix * maxTiles * sizeof(uint32_t)) != cudaSuccess ||
      cudaMalloc(&c->pos4, newCap * sizeof(double4)) != cudaSuccess ||
      cudaMalloc(&c->blockSums, (scanBlocks + 1) * sizeof(uint32_t)) != cudaSuccess) {
    cudaGetLastError();
    return fail(c, LADDS_ERR_ALLOC, "device allocation failed (sort counts)");
  }
  c->cap = newCap;
  c->orderValid = false;
  dropGraphs(c);
  return LADDS_OK;
}

int ensurePairCapacity(ladds_gpu_ctx *c, size_t need) {
  if (need <= c->pairCap) return LADDS_OK;
  size_t newCap = std::max<size_t>(need + need / 2, 1);
  ladds_pair *p = nullptr;
  if (cudaMalloc(&p, newCap * sizeof(ladds_pair)) != cudaSuccess) {
    cudaGetLastError();
    return fail(c, LADDS_ERR_ALLOC, "device allocation failed (pair buffer)");
  }
  if (c->dPairs) cudaFree(c->dPairs);
  c->dPairs = p;
  c->pairCap = newCap;
  dropGraphs(c);
  return LADDS_OK;
}

cudaEvent_t takeEvent(ladds_gpu_ctx *c) {
  if (!c->eventPool.empty()) {
    cudaEvent_t e = c->eventPool.back();
    c->eventPool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

struct PhaseScope {
  ladds_gpu_ctx *c;
  int phase;
  cudaEvent_t a = nullptr;
  PhaseScope(ladds_gpu_ctx *c_, int ph) : c(c_), phase(ph) {
    if (c->profiling) {
      a = takeEvent(c);
      cudaEventRecord(a, c->st);
    }
  }
  ~PhaseScope() {
    if (c->profiling) {
      cudaEvent_t b = takeEvent(c);
      cudaEventRecord(b, c->st);
      c->events.emplace_back(phase, a, b);
    }
  }
};

void collectTimes(ladds_gpu_ctx *c) {
  for (auto &t : c->events) {
    float ms = 0;
    cudaEventElapsedTime(&ms, std::get<1>(t), std::get<2>(t));
    switch (std::get<0>(t)) {
      case kPhProp:
        c->times.propagateMs += ms;
        c->times.propagateLaunches++;
        break;
      case kPhSort:
        c->times.sortMs += ms;
        c->times.sortLaunches++;
        break;
      case kPhCell:
        c->times.cellMs += ms;
        c->times.cellLaunches++;
        break;
      default:
        c->times.scanMs += ms;
        c->times.scanLaunches++;
        break;
    }
    c->eventPool.push_back(std::get<1>(t));
    c->eventPool.push_back(std::get<2>(t));
  }
  c->events.clear();
}

// ----- pipeline pieces (all enqueue on c->st; no synchronisation) -----

cudaError_t enqueueEphemeris(ladds_gpu_ctx *c, int nSteps) {
  const int threads = 3 * nSteps;
  k_ephemeris_dev<<<blocksFor(threads, 128), 128, 0, c->st>>>(c->dEph, nSteps, c->dIter, c->cfg.startTime,
                                                                c->cfg.deltaT, c->pc.hc1, c->pc.hc2,
                                                                c->cfg.epochJD, c->theta0);
  return cudaMemcpyToSymbolAsync(c_eph, c->dEph, (size_t)threads * sizeof(EphEntry), 0, cudaMemcpyDeviceToDevice,
                                 c->st);
}

void enqueuePropagate(ladds_gpu_ctx *c, int nSteps, bool keys) {
  if (c->n == 0) {
    k_advance<<<1, 32, 0, c->st>>>(c->dIter, nSteps);
    return;
  }
  PhaseScope ps(c, kPhProp);
  const int b = c->cfg.propagateBlock > 0 ? c->cfg.propagateBlock : 256;
  const int g = blocksFor(c->n, b);
  const bool split = c->cfg.precision == LADDS_PRECISION_SPLIT;
  if (split) {
    if (keys)
      k_propagate<true, true><<<g, b, 0, c->st>>>(c->cur, (int)c->n, nSteps, c->pc, c->grid, c->keys0, c->dStatus);
    else
      k_propagate<true, false><<<g, b, 0, c->st>>>(c->cur, (int)c->n, nSteps, c->pc, c->grid, c->keys0, c->dStatus);
  } else {
    if (keys)
      k_propagate<false, true><<<g, b, 0, c->st>>>(c->cur, (int)c->n, nSteps, c->pc, c->grid, c->keys0, c->dStatus);
    else
      k_propagate<false, false><<<g, b, 0, c->st>>>(c->cur, (int)c->n, nSteps, c->pc, c->grid, c->keys0,
                                                     c->dStatus);
  }
  k_advance<<<1, 32, 0, c->st>>>(c->dIter, nSteps);
}

// keys0 holds the keys of c->cur in current order -> sortedKeys / perm
void enqueueSort(ladds_gpu_ctx *c) {
  PhaseScope ps(c, kPhSort);
  const int n = (int)c->n;
  const int numTiles = blocksFor(c->n, kSortTile);
  const int passes = std::max(1, (int)((c->grid.keyBits + 7) / 8));
  const uint32_t *kin = c->keys0, *vin = nullptr;
  uint32_t *kout = c->keys1, *vout = c->vals1;
  for (int p = 0; p < passes; ++p) {
    const int shift = 8 * p;
    k_radix_hist<<<numTiles, kSortThreads, 0, c->st>>>(kin, n, shift, c->counts, numTiles);
    k_radix_scan_digit<<<kRadix, kSortThreads, 0, c->st>>>(c->counts, numTiles, c->totals);
    k_radix_scatter<<<numTiles, kSortThreads, 0, c->st>>>(kin, vin, kout, vout, n, shift, c->counts, c->totals,
                                                          numTiles, c->dStatus);
    kin = kout;
    vin = vout;
    kout = (kout == c->keys1) ? c->keys0 : c->keys1;
    vout = (vout == c->vals1) ? c->vals0 : c->vals1;
  }
  c->sortedKeys = const_cast<uint32_t *>(kin);
  c->perm = const_cast<uint32_t *>(vin);
}

void enqueueCells(ladds_gpu_ctx *c) {
  PhaseScope ps(c, kPhCell);
  k_permute<<<blocksFor(c->n, 256), 256, 0, c->st>>>(c->cur, c->alt, c->perm, (int)c->n, c->pos4, c->dStatus);
  std::swap(c->cur, c->alt);
  k_row_start<<<blocksFor((size_t)c->nRows + 1, 256), 256, 0, c->st>>>(c->sortedKeys, (int)c->n,
                                                                         (uint32_t)c->grid.n[0], c->nRows,
                                                                         c->rowStart);
}

void enqueueScan(ladds_gpu_ctx *c, double dtScan, int64_t iterOffset) {
  PhaseScope ps(c, kPhScan);
  ScanConsts sc = c->sc;
  sc.dt = dtScan;
  const int b = c->cfg.scanBlock > 0 ? c->cfg.scanBlock : 128;
  k_pair_scan<<<blocksFor(c->n, b), b, 0, c->st>>>(c->cur, c->pos4, (int)c->n, c->sortedKeys, c->rowStart, c->grid, sc,
                                                    c->dIter, iterOffset, c->dPairs, c->dCount,
                                                    (unsigned long long)c->pairCap);
}

void enqueueIteration(ladds_gpu_ctx *c, bool scan, int k) {
  enqueueEphemeris(c, 1);
  enqueuePropagate(c, 1, scan);
  if (scan && c->n) {
    enqueueSort(c);
    enqueueCells(c);
    enqueueScan(c, c->cfg.deltaT * (double)k, -1);  // records carry the iteration just integrated
  }
}

int syncAndStatus(ladds_gpu_ctx *c) {
  CK(cudaStreamSynchronize(c->st));
  CK(cudaGetLastError());
  unsigned status = 0;
  CK(cudaMemcpy(&status, c->dStatus, sizeof(unsigned), cudaMemcpyDeviceToHost));
  if (status) CK(cudaMemset(c->dStatus, 0, sizeof(unsigned)));
  if (status & 4u) return fail(c, LADDS_ERR_DEVICE_CHECK, "a device-side index check failed (sort / gather)");
  if (status & 1u) return fail(c, LADDS_ERR_NONFINITE, "a position or velocity became NaN/Inf during propagation");
  return LADDS_OK;
}

bool pairLess(const ladds_pair &a, const ladds_pair &b) {
  if (a.step != b.step) return a.step < b.step;
  if (a.idA != b.idA) return a.idA < b.idA;
  if (a.idB != b.idB) return a.idB < b.idB;
  if (a.slotA != b.slotA) return a.slotA < b.slotA;
  return a.slotB < b.slotB;
}

int validateArrays(ladds_gpu_ctx *c, size_t n, const double *const *arrs, int nArr, const int8_t *activity) {
  for (int a = 0; a < nArr; ++a)
    if (n && !arrs[a]) return fail(c, LADDS_ERR_INVALID_ARG, "null array pointer");
  for (int a = 0; a < 6; ++a)
    for (size_t i = 0; i < n; ++i)
      if (!std::isfinite(arrs[a][i])) return fail(c, LADDS_ERR_INVALID_ARG, "non-finite position or velocity");
  if (activity)
    for (size_t i = 0; i < n; ++i)
      if (activity[i] < 0 || activity[i] > 2) return fail(c, LADDS_ERR_INVALID_ARG, "activity state out of range");
  return LADDS_OK;
}

int writeArrays(ladds_gpu_ctx *c, size_t offset, size_t n, const double *x, const double *y, const double *z,
                const double *vx, const double *vy, const double *vz, const double *radius, const double *aom,
                const double *bcInv, const uint64_t *id, const uint64_t *parentId, const int8_t *activity) {
  if (!n) return LADDS_OK;
  const double *src[] = {x, y, z, vx, vy, vz, aom, bcInv, radius};
  double *dst[] = {c->cur.x, c->cur.y, c->cur.z, c->cur.vx, c->cur.vy, c->cur.vz, c->cur.aom, c->cur.bc,
                   c->cur.radius};
  for (int k = 0; k < 9; ++k)
    CK(cudaMemcpyAsync(dst[k] + offset, src[k], n * sizeof(double), cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->cur.id + offset, id, n * sizeof(uint64_t), cudaMemcpyHostToDevice, c->st));
  std::vector<uint64_t> par;
  if (!parentId) par.assign(n, UINT64_MAX);
  CK(cudaMemcpyAsync(c->cur.parent + offset, parentId ? parentId : par.data(), n * sizeof(uint64_t),
                     cudaMemcpyHostToDevice, c->st));
  std::vector<uint32_t> tags(n);
  for (size_t i = 0; i < n; ++i) tags[i] = makeTag((uint32_t)(offset + i), activity ? activity[i] : 0, false);
  CK(cudaMemcpyAsync(c->cur.tag + offset, tags.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  return LADDS_OK;
}

int buildGrid(ladds_gpu_ctx *c) {
  const ladds_gpu_config &f = c->cfg;
  // default edge: just above the cutoff, so that the neighbour reach is one cell
  double cell = f.cellSize > 0 ? f.cellSize : f.cutoff * (1.0 + 1e-6);
  const double minCell = std::max(f.cutoff * 1e-3, 1e-9);
  if (!(cell > minCell)) cell = minCell;
  for (int d = 0; d < 3; ++d)
    if (!(f.boxMax[d] > f.boxMin[d]) || !std::isfinite(f.boxMax[d] - f.boxMin[d]))
      return fail(c, LADDS_ERR_INVALID_ARG, "boxMax must exceed boxMin");
  GridDesc g{};
  uint64_t total = 0;
  // coarsen until the keys fit 32 bits and no axis exceeds 65535 cells
  for (;;) {
    g.cellSize = cell;
    g.invCell = 1.0 / cell;
    total = 1;
    bool ok = true;
    for (int d = 0; d < 3; ++d) {
      g.boxMin[d] = f.boxMin[d];
      double cells = std::ceil((f.boxMax[d] - f.boxMin[d]) * g.invCell);
      if (!(cells >= 1.0)) cells = 1.0;
      if (cells > 65535.0) ok = false;
      g.n[d] = (int32_t)std::min(cells, 65535.0);
      total *= (uint64_t)g.n[d];
    }
    if (ok && total <= (1ull << 32)) break;
    cell *= 1.25;
  }
  int32_t r = (int32_t)std::ceil(f.cutoff * (1.0 + 1e-9) * g.invCell);
  if (r < 1) r = 1;
  while ((double)r * cell < f.cutoff * (1.0 + 1e-9)) ++r;
  g.reach = r;
  uint32_t bits = 0;
  while (bits < 32 && ((total - 1) >> bits) != 0) ++bits;
  g.keyBits = bits;
  c->grid = g;
  c->nRows = (uint32_t)((uint64_t)g.n[1] * (uint64_t)g.n[2]);
  return LADDS_OK;
}

}  // namespace

extern "C" {

int ladds_gpu_abi_version(void) { return LADDS_GPU_ABI_VERSION; }

void ladds_gpu_config_default(ladds_gpu_config *f) {
  if (!f) return;
  std::memset(f, 0, sizeof(*f));
  f->deltaT = 10.0;
  f->componentMask =
      LADDS_PROP_KEP | LADDS_PROP_J2 | LADDS_PROP_C22 | LADDS_PROP_S22 | LADDS_PROP_SRP | LADDS_PROP_DRAG;
  f->epochJD = 2459580.5;  // 2022-01-01 00:00 UTC (cfg/default_cfg.yaml:9)
  f->startTime = 0.0;
  f->cutoff = 80.0;
  f->collisionDistanceFactor = 1.0;
  f->minDetectionRadius = 0.05;
  f->evasionCutoff = 0.1;
  f->conjunctionThreshold = 0.1;
  f->nearThresholdRel = 1e-9;
  f->precision = LADDS_PRECISION_FP64;
  f->timestepsPerCollisionDetection = 1;
  f->cellSize = 0.0;
  for (int d = 0; d < 3; ++d) {
    f->boxMin[d] = -10000.0;
    f->boxMax[d] = 10000.0;
  }
  f->device = 0;
  f->propagateBlock = 256;
  f->scanBlock = 128;
  f->useGraphs = 1;
  f->pairCapacity = 0;
}

const char *ladds_gpu_last_error(const ladds_gpu_ctx *c) { return c ? c->err.c_str() : "null context"; }

int ladds_gpu_create(const ladds_gpu_config *f, ladds_gpu_ctx **out) {
  if (!f || !out) return LADDS_ERR_INVALID_ARG;
  *out = nullptr;
  if (!(f->deltaT != 0.0 && std::isfinite(f->deltaT)) || !(f->cutoff > 0) || f->timestepsPerCollisionDetection < 1 ||
      (f->precision != LADDS_PRECISION_FP64 && f->precision != LADDS_PRECISION_SPLIT) ||
      (f->componentMask & ~LADDS_PROP_ALL) || !(f->nearThresholdRel >= 0))
    return LADDS_ERR_INVALID_ARG;
  if (f->propagateBlock < 0 || f->propagateBlock > 256 || (f->propagateBlock % 32) || f->scanBlock < 0 ||
      f->scanBlock > 128 || (f->scanBlock % 32))
    return LADDS_ERR_INVALID_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
    cudaGetLastError();
    return LADDS_ERR_NO_DEVICE;
  }
  if (f->device < 0 || f->device >= ndev) return LADDS_ERR_NO_DEVICE;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, f->device) != cudaSuccess || prop.major < 10) return LADDS_ERR_NO_DEVICE;
  ladds_gpu_ctx *c = new ladds_gpu_ctx();
  c->cfg = *f;
  c->dev = f->device;
  int rc = buildGrid(c);
  if (rc) {
    delete c;
    return rc;
  }
  const double dt = f->deltaT;
  c->pc.hc1 = kYoshidaC1 * dt;
  c->pc.hc2 = kYoshidaC2 * dt;
  c->pc.hd1 = kYoshidaD1 * dt;
  c->pc.hd2 = kYoshidaD2 * dt;
  c->pc.mask = f->componentMask;
  c->sc.cutoffSq = f->cutoff * f->cutoff;
  c->sc.dt = dt;
  c->sc.factor = f->collisionDistanceFactor / 1000.;
  c->sc.minDetectionRadius = f->minDetectionRadius;
  c->sc.evasionSq = f->evasionCutoff * f->evasionCutoff;
  c->sc.conjSq = f->conjunctionThreshold * f->conjunctionThreshold;
  c->sc.nearRel = f->nearThresholdRel;
  c->theta0 = gmstIAU1982(f->epochJD);
  if (cudaSetDevice(c->dev) != cudaSuccess || cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&c->rowStart, ((size_t)c->nRows + 1) * sizeof(uint32_t)) != cudaSuccess ||
      cudaMalloc(&c->totals, kRadix * sizeof(uint32_t)) != cudaSuccess ||
      cudaMalloc(&c->dCount, sizeof(unsigned long long)) != cudaSuccess ||
      cudaMalloc(&c->dStatus, sizeof(unsigned)) != cudaSuccess ||
      cudaMalloc(&c->dEph, 3 * kMaxEphSteps * sizeof(EphEntry)) != cudaSuccess ||
      cudaMalloc(&c->dIter, sizeof(int64_t)) != cudaSuccess) {
    cudaGetLastError();
    ladds_gpu_destroy(c);
    return LADDS_ERR_ALLOC;
  }
  cudaMemset(c->dStatus, 0, sizeof(unsigned));
  cudaMemset(c->dCount, 0, sizeof(unsigned long long));
  cudaMemset(c->dIter, 0, sizeof(int64_t));
  cudaEventCreate(&c->callStart);
  cudaEventCreate(&c->callEnd);
  rc = ensurePairCapacity(c, f->pairCapacity ? (size_t)f->pairCapacity : (size_t)1 << 16);
  if (rc) {
    ladds_gpu_destroy(c);
    return rc;
  }
  if (cudaDeviceSynchronize() != cudaSuccess) {
    cudaGetLastError();
    ladds_gpu_destroy(c);
    return LADDS_ERR_CUDA;
  }
  *out = c;
  return LADDS_OK;
}

int ladds_gpu_destroy(ladds_gpu_ctx *c) {
  if (!c) return LADDS_ERR_INVALID_ARG;
  cudaSetDevice(c->dev);
  if (c->st) cudaStreamSynchronize(c->st);
  dropGraphs(c);
  freeBuffers(c);
  void *ptrs[] = {c->rowStart, c->totals, c->dCount, c->dStatus, c->dEph, c->dIter, c->dPairs};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  for (auto &t : c->events) {
    cudaEventDestroy(std::get<1>(t));
    cudaEventDestroy(std::get<2>(t));
  }
  for (auto e : c->eventPool) cudaEventDestroy(e);
  if (c->callStart) cudaEventDestroy(c->callStart);
  if (c->callEnd) cudaEventDestroy(c->callEnd);
  if (c->st) cudaStreamDestroy(c->st);
  delete c;
  return LADDS_OK;
}

int ladds_gpu_upload(ladds_gpu_ctx *c, size_t n, const double *x, const double *y, const double *z,
                     const double *vx, const double *vy, const double *vz, const double *radius, const double *aom,
                     const double *bcInv, const uint64_t *id, const uint64_t *parentId, const int8_t *activity) {
  if (!c) return LADDS_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g_deviceMutex[c->dev & 63]);
  const double *arrs[] = {x, y, z, vx, vy, vz, radius, aom, bcInv};
  int rc = validateArrays(c, n, arrs, 9, activity);
  if (rc) return rc;
  if (n && !id) return fail(c, LADDS_ERR_INVALID_ARG, "null id array");
  CK(cudaSetDevice(c->dev));
  rc = ensureCapacity(c, n);
  if (rc) return rc;
  c->n = 0;
  rc = writeArrays(c, 0, n, x, y, z, vx, vy, vz, radius, aom, bcInv, id, parentId, activity);
  if (rc) return rc;
  c->n = n;
  c->orderValid = false;
  dropGraphs(c);
  return LADDS_OK;
}

int ladds_gpu_append(ladds_gpu_ctx *c, size_t n, const double *x, const double *y, const double *z,
                     const double *vx, const double *vy, const double *vz, const double *radius, const double *aom,
                     const double *bcInv, const uint64_t *id, const uint64_t *parentId, const int8_t *activity) {
  if (!c) return LADDS_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g_deviceMutex[c->dev & 63]);
  const double *arrs[] = {x, y, z, vx, vy, vz, radius, aom, bcInv};
  int rc = validateArrays(c, n, arrs, 9, activity);
  if (rc) return rc;
  if (n && !id) return fail(c, LADDS_ERR_INVALID_ARG, "null id array");
  if (!n) return LADDS_OK;
  CK(cudaSetDevice(c->dev));
  rc = ensureCapacity(c, c->n + n);
  if (rc) return rc;
  rc = writeArrays(c, c->n, n, x, y, z, vx, vy, vz, radius, aom, bcInv, id, parentId, activity);
  if (rc) return rc;
  c->n += n;
  c->orderValid = false;
  dropGraphs(c);
  return LADDS_OK;
}

int ladds_gpu_download(ladds_gpu_ctx *c, size_t cap, size_t *nOut, double *x, double *y, double *z, double *vx,
                       double *vy, double *vz, double *radius, double *aom, double *bcInv, uint64_t *id,
                       uint64_t *parentId, int8_t *activity) {
  if (!c) return LADDS_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g_deviceMutex[c->dev & 63]);
  if (nOut) *nOut = c->n;
  if (cap < c->n) return fail(c, LADDS_ERR_CAPACITY, "download buffer smaller than the population");
  if (!c->n) return LADDS_OK;
  CK(cudaSetDevice(c->dev));
  const int g = blocksFor(c->n, 256);
  const double *src[] = {c->cur.x, c->cur.y, c->cur.z, c->cur.vx, c->cur.vy, c->cur.vz, c->cur.radius, c->cur.aom,
                         c->cur.bc};
  double *dst[] = {x, y, z, vx, vy, vz, radius, aom, bcInv};
  for (int k = 0; k < 9; ++k) {
    if (!dst[k]) continue;
    k_unpermute_f64<<<g, 256, 0, c->st>>>(src[k], c->cur.tag, (int)c->n, c->alt.x);
    CK(cudaMemcpyAsync(dst[k], c->alt.x, c->n * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
  }
  const uint64_t *usrc[] = {c->cur.id, c->cur.parent};
  uint64_t *udst[] = {id, parentId};
  for (int k = 0; k < 2; ++k) {
    if (!udst[k]) continue;
    k_unpermute_u64<<<g, 256, 0, c->st>>>(usrc[k], c->cur.tag, (int)c->n, c->alt.id);
    CK(cudaMemcpyAsync(udst[k], c->alt.id, c->n * sizeof(uint64_t), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
  }
  if (activity) {
    k_unpermute_act<<<g, 256, 0, c->st>>>(c->cur.tag, (int)c->n, (int8_t *)c->alt.tag);
    CK(cudaMemcpyAsync(activity, c->alt.tag, c->n, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
  }
  CK(cudaGetLastError());
  return LADDS_OK;
}

int ladds_gpu_set_state(ladds_gpu_ctx *c, size_t n, const double *x, const double *y, const double *z,
                        const double *vx, const double *vy, const double *vz) {
  if (!c) return LADDS_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g_deviceMutex[c->dev & 63]);
  if (n != c->n) return fail(c, LADDS_ERR_INVALID_ARG, "set_state: n differs from the population size");
  const double *src[] = {x, y, z, vx, vy, vz};
  for (int k = 0; k < 6; ++k)
    if (n && !src[k]) return fail(c, LADDS_ERR_INVALID_ARG, "null array pointer");
  if (!n) return LADDS_OK;
  CK(cudaSetDevice(c->dev));
  double *dst[] = {c->cur.x, c->cur.y, c->cur.z, c->cur.vx, c->cur.vy, c->cur.vz};
  double *stage[] = {c->alt.x, c->alt.y, c->alt.z, c->alt.vx, c->alt.vy, c->alt.vz};
  const int g = blocksFor(n, 256);
  for (int k = 0; k < 6; ++k) {
    CK(cudaMemcpyAsync(stage[k], src[k], n * sizeof(double), cudaMemcpyHostToDevice, c->st));
    k_permute_from_slots_f64<<<g, 256, 0, c->st>>>(stage[k], c->cur.tag, (int)n, dst[k]);
  }
  CK(cudaStreamSynchronize(c->st));
  CK(cudaGetLastError());
  return LADDS_OK;
}

int ladds_gpu_get_state(ladds_gpu_ctx *c, size_t n, double *x, double *y, double *z, double *vx, double *vy,
                        double *vz) {
  if (!c) return LADDS_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g_deviceMutex[c->dev & 63]);
  if (n < c->n) return fail(c, LADDS_ERR_CAPACITY, "get_state: buffer smaller than the population");
  if (!c->n) return LADDS_OK;
  CK(cudaSetDevice(c->dev));
  const double *src[] = {c->cur.x, c->cur.y, c->cur.z, c->cur.vx, c->cur.vy, c->cur.vz};
  double *stage[] = {c->alt.x, c->alt.y, c->alt.z, c->alt.vx, c->alt.vy, c->alt.vz};
  double *dst[] = {x, y, z, vx, vy, vz};
  const int g = blocksFor(c->n, 256);
  for (int k = 0; k < 6; ++k) {
    if (!dst[k]) continue;
    k_unpermute_f64<<<g, 256, 0, c->st>>>(src[k], c->cur.tag, (int)c->n, stage[k]);
    CK(cudaMemcpyAsync(dst[k], stage[k], c->n * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  }
  CK(cudaStreamSynchronize(c->st));
  CK(cudaGetLastError());
  return LADDS_OK;
}

int ladds_gpu_size(const ladds_gpu_ctx *c, size_t *n) {
  if (!c || !n) return LADDS_ERR_INVALID_ARG;
  *n = c->n;
  return LADDS_OK;
}

int ladds_gpu_iteration(const ladds_gpu_ctx *c, int64_t *it) {
  if (!c || !it) return LADDS_ERR_INVALID_ARG;
  *it = c->hostIter;
  return LADDS_OK;
}

int ladds_gpu_set_iteration(ladds_gpu_ctx *c, int64_t it) {
  if (!c || it < 0) return LADDS_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g_deviceMutex[c->dev & 63]);
  CK(cudaSetDevice(c->dev));
  CK(cudaMemcpyAsync(c->dIter, &it, sizeof(int64_t), cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  c->hostIter = it;
  return LADDS_OK;
}

int ladds_gpu_set_profiling(ladds_gpu_ctx *c, int enable) {
  if (!c) return LADDS_ERR_INVALID_ARG;
  c->profiling = enable != 0;
  std::memset(&c->times, 0, sizeof(c->times));
  return LADDS_OK;
}

int ladds_gpu_phase_times(ladds_gpu_ctx *c, ladds_phase_times *t) {
  if (!c || !t) return LADDS_ERR_INVALID_ARG;
  *t = c->times;
  t->totalMs = t->propagateMs + t->sortMs + t->cellMs + t->scanMs;
  return LADDS_OK;
}

int ladds_gpu_integrate(ladds_gpu_ctx *c, int steps) {
  if (!c || steps < 0) return LADDS_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g_deviceMutex[c->dev & 63]);
  CK(cudaSetDevice(c->dev));
  int left = steps;
  while (left > 0) {
    const int chunk = std::min(left, kMaxEphSteps);
    CK(enqueueEphemeris(c, chunk));
    enqueuePropagate(c, chunk, false);
    left -= chunk;
  }
  const int rc = syncAndStatus(c);
  collectTimes(c);
  c->hostIter += steps;
  c->orderValid = false;
  return rc;
}

int ladds_gpu_conjunctions(ladds_gpu_ctx *c, double dtScan, ladds_pair *out, size_t cap, size_t *nOut,
                           size_t *nCollisions, size_t *nEvasions, size_t *nConjunctions) {
  if (!c || !nOut || !std::isfinite(dtScan)) return LADDS_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g_deviceMutex[c->dev & 63]);
  CK(cudaSetDevice(c->dev));
  std::vector<ladds_pair> recs;
  if (c->n) {
    for (int attempt = 0; attempt < 4; ++attempt) {
      CK(cudaMemsetAsync(c->dCount, 0, sizeof(unsigned long long), c->st));
      k_cell_keys<<<blocksFor(c->n, 256), 256, 0, c->st>>>(c->cur.x, c->cur.y, c->cur.z, (int)c->n, c->grid,
                                                            c->keys0);
      enqueueSort(c);
      enqueueCells(c);
      enqueueScan(c, dtScan, -1);  // records carry the index of the last integrated iteration
      int rc = syncAndStatus(c);
      collectTimes(c);
      if (rc) return rc;
      unsigned long long cnt = 0;
      CK(cudaMemcpy(&cnt, c->dCount, sizeof(cnt), cudaMemcpyDeviceToHost));
      if (cnt <= c->pairCap) {
        recs.resize(cnt);
        if (cnt) CK(cudaMemcpy(recs.data(), c->dPairs, cnt * sizeof(ladds_pair), cudaMemcpyDeviceToHost));
        break;
      }
      rc = ensurePairCapacity(c, (size_t)cnt);
      if (rc) return rc;
    }
    c->orderValid = true;
  }
  std::sort(recs.begin(), recs.end(), pairLess);
  size_t nc = 0, ne = 0, nj = 0;
  for (const auto &p : recs) {
    nc += (p.flags & LADDS_PAIR_COLLISION) != 0;
    ne += (p.flags & LADDS_PAIR_EVASION) != 0;
    nj += (p.flags & LADDS_PAIR_CONJUNCTION) != 0;
  }
  if (nCollisions) *nCollisions = nc;
  if (nEvasions) *nEvasions = ne;
  if (nConjunctions) *nConjunctions = nj;
  *nOut = recs.size();
  if (recs.size() > cap || (!out && !recs.empty()))
    return fail(c, LADDS_ERR_CAPACITY, "output buffer too small for the conjunction records");
  if (!recs.empty()) std::memcpy(out, recs.data(), recs.size() * sizeof(ladds_pair));
  return LADDS_OK;
}

int ladds_gpu_step(ladds_gpu_ctx *c, int iterations, ladds_pair *out, size_t cap, size_t *nOut,
                   ladds_step_stats *stats) {
  if (!c || iterations < 0 || !nOut) return LADDS_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g_deviceMutex[c->dev & 63]);
  CK(cudaSetDevice(c->dev));
  if (stats) std::memset(stats, 0, sizeof(*stats));
  const int k = c->cfg.timestepsPerCollisionDetection;
  int scans = 0;
  for (int i = 0; i < iterations; ++i) scans += ((c->hostIter + i) % k) == 0;
  // snapshot of the call's start state: the call is re-run after a device
  // pair-buffer overflow and undone when the caller's buffer is too small
  CK(copyState(c->cur, c->snap, c->n, c->st));
  const int64_t startIter = c->hostIter;
  auto rollBack = [&]() -> int {
    CK(copyState(c->snap, c->cur, c->n, c->st));
    CK(cudaMemcpyAsync(c->dIter, &startIter, sizeof(int64_t), cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    c->hostIter = startIter;
    c->orderValid = false;
    return LADDS_OK;
  };
  unsigned long long cnt = 0;
  int retries = 0;
  for (;;) {
    CK(cudaMemsetAsync(c->dCount, 0, sizeof(unsigned long long), c->st));
    CK(cudaEventRecord(c->callStart, c->st));
    const bool graph = c->cfg.useGraphs && !c->profiling && iterations > 1;
    if (graph) {
      const auto key =
          std::make_tuple(iterations, (int)(c->hostIter % k), c->cur.x == c->homeX ? 0 : 1, c->n, c->pairCap);
      auto it = c->graphs.find(key);
      if (it == c->graphs.end()) {
        // capture performs the host-side buffer swaps of the batch
        CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
        for (int i = 0; i < iterations; ++i) enqueueIteration(c, ((c->hostIter + i) % k) == 0, k);
        cudaGraph_t gr = nullptr;
        CK(cudaStreamEndCapture(c->st, &gr));
        cudaGraphExec_t ex = nullptr;
        const cudaError_t ie = cudaGraphInstantiate(&ex, gr, 0);
        cudaGraphDestroy(gr);
        CK(ie);
        it = c->graphs.emplace(key, ex).first;
      } else if (scans) {
        // a replay performs the swaps of the captured batch
        if (scans % 2 == 1) std::swap(c->cur, c->alt);
        const int passes = std::max(1, (int)((c->grid.keyBits + 7) / 8));
        c->sortedKeys = (passes % 2) ? c->keys1 : c->keys0;
        c->perm = (passes % 2) ? c->vals1 : c->vals0;
      }
      CK(cudaGraphLaunch(it->second, c->st));
    } else {
      for (int i = 0; i < iterations; ++i) enqueueIteration(c, ((c->hostIter + i) % k) == 0, k);
    }
    CK(cudaEventRecord(c->callEnd, c->st));
    int rc = syncAndStatus(c);
    collectTimes(c);
    if (rc) {
      const int rb = rollBack();
      return rb ? rb : rc;
    }
    CK(cudaMemcpy(&cnt, c->dCount, sizeof(cnt), cudaMemcpyDeviceToHost));
    if (cnt <= c->pairCap) break;
    // device pair buffer overflowed: grow it, roll back, run the batch again
    if (++retries > 4) {
      rollBack();
      return fail(c, LADDS_ERR_CAPACITY, "device pair buffer kept overflowing");
    }
    rc = rollBack();
    if (rc) return rc;
    rc = ensurePairCapacity(c, (size_t)cnt);
    if (rc) return rc;
  }
  float ms = 0;
  cudaEventElapsedTime(&ms, c->callStart, c->callEnd);
  std::vector<ladds_pair> recs(cnt);
  if (cnt) CK(cudaMemcpy(recs.data(), c->dPairs, cnt * sizeof(ladds_pair), cudaMemcpyDeviceToHost));
  std::sort(recs.begin(), recs.end(), pairLess);
  *nOut = recs.size();
  if (recs.size() > cap || (!out && !recs.empty())) {
    const int rb = rollBack();
    if (rb) return rb;
    return fail(c, LADDS_ERR_CAPACITY, "output buffer too small for the conjunction records");
  }
  if (!recs.empty()) std::memcpy(out, recs.data(), recs.size() * sizeof(ladds_pair));
  c->hostIter += iterations;
  if (scans) c->orderValid = true;
  if (stats) {
    stats->iterations = (uint64_t)iterations;
    stats->scans = (uint64_t)scans;
    stats->records = cnt;
    stats->retries = (uint64_t)retries;
    stats->deviceMs = ms;
    for (const auto &p : recs) {
      stats->collisions += (p.flags & LADDS_PAIR_COLLISION) != 0;
      stats->evasions += (p.flags & LADDS_PAIR_EVASION) != 0;
      stats->conjunctions += (p.flags & LADDS_PAIR_CONJUNCTION) != 0;
    }
  }
  return LADDS_OK;
}

int ladds_gpu_cell_order(ladds_gpu_ctx *c, size_t cap, size_t *n, uint32_t *keys, uint32_t *slots) {
  if (!c || !n) return LADDS_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g_deviceMutex[c->dev & 63]);
  if (!c->orderValid) return fail(c, LADDS_ERR_STATE, "no conjunction scan since the last change of the state");
  *n = c->n;
  if (cap < c->n) return fail(c, LADDS_ERR_CAPACITY, "buffer smaller than the population");
  if (!c->n) return LADDS_OK;
  CK(cudaSetDevice(c->dev));
  if (keys) CK(cudaMemcpy(keys, c->sortedKeys, c->n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
  if (slots) {
    std::vector<uint32_t> tags(c->n);
    CK(cudaMemcpy(tags.data(), c->cur.tag, c->n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < c->n; ++i) slots[i] = tagSlot(tags[i]);
  }
  return LADDS_OK;
}

int ladds_gpu_grid(const ladds_gpu_ctx *c, int32_t dims[3], int32_t *reach, double *cellSize) {
  if (!c) return LADDS_ERR_INVALID_ARG;
  if (dims)
    for (int d = 0; d < 3; ++d) dims[d] = c->grid.n[d];
  if (reach) *reach = c->grid.reach;
  if (cellSize) *cellSize = c->grid.cellSize;
  return LADDS_OK;
}

int ladds_gpu_clear_parents(ladds_gpu_ctx *c) {
  if (!c) return LADDS_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g_deviceMutex[c->dev & 63]);
  if (!c->n) return LADDS_OK;
  CK(cudaSetDevice(c->dev));
  k_clear_parents<<<blocksFor(c->n, 256), 256, 0, c->st>>>(c->cur.parent, (int)c->n);
  CK(cudaStreamSynchronize(c->st));
  CK(cudaGetLastError());
  return LADDS_OK;
}

int ladds_gpu_mark_deleted(ladds_gpu_ctx *c, const uint32_t *slots, size_t m) {
  if (!c || (m && !slots)) return LADDS_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g_deviceMutex[c->dev & 63]);
  if (!m || !c->n) return LADDS_OK;
  for (size_t i = 0; i < m; ++i)
    if (slots[i] >= c->n) return fail(c, LADDS_ERR_INVALID_ARG, "slot out of range");
  CK(cudaSetDevice(c->dev));
  std::vector<uint8_t> mark(c->n, 0);
  for (size_t i = 0; i < m; ++i) mark[slots[i]] = 1;
  uint8_t *dMark = reinterpret_cast<uint8_t *>(c->scratchA);
  CK(cudaMemcpyAsync(dMark, mark.data(), c->n, cudaMemcpyHostToDevice, c->st));
  k_mark_deleted<<<blocksFor(c->n, 256), 256, 0, c->st>>>(c->cur.tag, dMark, (int)c->n);
  CK(cudaStreamSynchronize(c->st));
  CK(cudaGetLastError());
  return LADDS_OK;
}

int ladds_gpu_remove_below(ladds_gpu_ctx *c, double minAltitude, size_t *nRemoved, uint64_t *removedIds,
                           size_t cap) {
  if (!c || !std::isfinite(minAltitude)) return LADDS_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g_deviceMutex[c->dev & 63]);
  if (nRemoved) *nRemoved = 0;
  if (!c->n) return LADDS_OK;
  CK(cudaSetDevice(c->dev));
  const int n = (int)c->n;
  const double crit = kREarth + minAltitude;  // Simulation.cpp:573
  const double critSq = crit * crit;           // Simulation.cpp:581
  uint32_t *keep = c->scratchA, *pos = c->scratchB, *aliveBySlot = c->scratchC, *newSlot = c->keys1;
  k_burnup_flags<<<blocksFor(n, 256), 256, 0, c->st>>>(c->cur.x, c->cur.y, c->cur.z, c->cur.tag, n, critSq, keep,
                                                        aliveBySlot);
  // exclusive scans: positions in the current order, new slot numbers in slot order
  auto exclusiveScan = [&](const uint32_t *in, uint32_t *outp) -> cudaError_t {
    const int nb = blocksFor((size_t)n, kScanBlock);
    k_scan_blocks<<<nb, kScanBlock, 0, c->st>>>(in, n, outp, c->blockSums);
    if (nb > 1) {
      // scan of block sums (nb <= 262144 for the 2^28 limit: two levels suffice up to 2^30)
      uint32_t *bs2 = c->vals1;
      const int nb2 = blocksFor((size_t)nb, kScanBlock);
      k_scan_blocks<<<nb2, kScanBlock, 0, c->st>>>(c->blockSums, nb, c->vals0, bs2);
      if (nb2 > 1) {
        k_scan_blocks<<<1, kScanBlock, 0, c->st>>>(bs2, nb2, c->keys0, bs2 + nb2 + 1);
        k_scan_add<<<nb2, kScanBlock, 0, c->st>>>(c->vals0, nb, c->keys0);
      }
      k_scan_add<<<nb, kScanBlock, 0, c->st>>>(outp, n, c->vals0);
    }
    return cudaGetLastError();
  };
  CK(exclusiveScan(keep, pos));
  CK(exclusiveScan(aliveBySlot, newSlot));
  k_compact<<<blocksFor(n, 256), 256, 0, c->st>>>(c->cur, c->alt, keep, pos, newSlot, n);
  CK(cudaStreamSynchronize(c->st));
  CK(cudaGetLastError());
  std::vector<uint32_t> hKeep(n);
  CK(cudaMemcpy(hKeep.data(), keep, n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
  size_t kept = 0;
  for (int i = 0; i < n; ++i) kept += hKeep[i];
  const size_t removed = c->n - kept;
  if (removedIds && removed) {
    std::vector<uint64_t> ids(n);
    CK(cudaMemcpy(ids.data(), c->cur.id, n * sizeof(uint64_t), cudaMemcpyDeviceToHost));
    size_t w = 0;
    for (int i = 0; i < n && w < cap; ++i)
      if (!hKeep[i]) removedIds[w++] = ids[i];
  }
  std::swap(c->cur, c->alt);
  c->n = kept;
  if (nRemoved) *nRemoved = removed;
  c->orderValid = false;
  dropGraphs(c);
  return LADDS_OK;
}

}  // extern "C"
