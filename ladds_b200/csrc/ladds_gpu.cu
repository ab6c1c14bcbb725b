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
#include "cell_sort.cuh"
#include "pair_scan.cuh"
#include "propagate.cuh"
#include "adjoint.cuh"
#include "insert.cuh"
#include "population.h"

using namespace ladds;

namespace {

// c_eph is per device: calls on one device are serialised.
std::mutex g_deviceMutex[64];

__global__ void k_advance(int64_t *iter, int by) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *iter += by;
}
// also stores the chunk's first iteration in *iterBase (the scans' step index)
__global__ void k_ephemeris_dev(EphEntry *__restrict__ out, int nSteps, const int64_t *__restrict__ iterPtr,
                                int64_t *__restrict__ iterBase, double t0, double dt, double hc1, double hc2,
                                double jdEpoch, double theta0) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) *iterBase = *iterPtr;
  if (i >= 3 * nSteps) return;
  const int st = i / 3, stage = i % 3;
  const double tn = t0 + (double)(*iterPtr + st) * dt;
  double tau = tn + hc1;
  if (stage >= 1) tau += hc2;
  if (stage >= 2) tau += hc2;
  ephemeris(jdEpoch, theta0, tau, out[i]);
}

inline int blocksFor(size_t n, int b) { return (int)((n + (size_t)b - 1) / (size_t)b); }

enum Phase { kPhProp, kPhBucket, kPhRowsort, kPhPermute, kPhCandidates, kPhEvaluate };

// ladds_gpu_step_host moves the state in at most this many chunks, each at
// least kHostChunkMin objects (smaller copies cost more than they overlap)
constexpr int kHostChunks = 4;
constexpr size_t kHostChunkMin = (size_t)1 << 17;

}  // namespace

struct ladds_gpu_ctx {
  ladds_gpu_config cfg{};
  GridDesc grid{};
  PropConsts pc{};
  ScanConsts sc{};
  double theta0 = 0;
  int dev = 0;
  cudaStream_t st = nullptr;   // main stream
  cudaStream_t st2 = nullptr;  // pair scans, overlapped with the next propagation
  cudaStream_t st3 = nullptr;  // device-to-host copies of ladds_gpu_step_host
  cudaEvent_t evCells = nullptr, evScan = nullptr;
  cudaEvent_t evXfer[7] = {};  // per-array hand-offs between copies and (un)permutes of set/get_state
  cudaEvent_t evPipe[3 * kHostChunks + 1] = {};  // chunk hand-offs of ladds_gpu_step_host
  double *pinStage = nullptr;  // pinned staging of ladds_gpu_step_host for pageable arrays (12 x pinCap)
  size_t pinCap = 0;
  std::vector<ladds_pair> pending;  // records of a ladds_gpu_step_host call whose buffer was too small
  int64_t *dIterBase = nullptr;  // first iteration of the chunk being run (device)
  size_t n = 0, cap = 0;
  DevState cur{}, alt{}, snap{};
  uint32_t *keys0 = nullptr, *keys1 = nullptr, *vals0 = nullptr, *vals1 = nullptr;
  uint32_t *sortedKeys = nullptr, *perm = nullptr;  // results of the last sort
  unsigned long long *sortRec = nullptr;  // (ix << 32 | slot) sort records of the bucket sort
  uint32_t *rowCounts = nullptr;          // objects per row (nRows + 1 used of 2 x (nRows + 1))
  uint32_t *longRows = nullptr, *longCount = nullptr;  // rows with more than 256 objects
  uint16_t *cellOff = nullptr;            // per row: offset of every cell inside the row (cellOffPitch entries)
  uint32_t *scanWs = nullptr;             // block sums of the exclusive scans
  float4 *posf = nullptr;                 // binary32 positions + rounding bound, cell order
  float4 *velf = nullptr;                 // binary32 velocities + radius of the cell order
  uint32_t *grp = nullptr;                // breakup group of the cell order (parent id, or kNoGroup)
  bool anyParent = false;                 // some object has a parent id: the scan writes and reads grp
  uint32_t *rowStart = nullptr;
  uint32_t nRows = 0;
  uint32_t *scratchA = nullptr, *scratchB = nullptr, *scratchC = nullptr, *blockSums = nullptr;
  ladds_pair *dPairs = nullptr;
  size_t pairCap = 0;
  unsigned long long *dCount = nullptr;
  uint2 *dCand = nullptr;  // candidate pairs (sorted indices) of the pair scan
  size_t candCap = 0;  // entries of each of the two candidate lists
  unsigned long long *dCandCount = nullptr;  // lengths of the candidate lists of the current scan
  unsigned long long *dCandNeed = nullptr;   // largest candidate count of the call
  unsigned *dStatus = nullptr;
  EphEntry *dEph = nullptr;
  int64_t *dIter = nullptr;
  int64_t hostIter = 0;
  bool orderValid = false;
  bool profiling = false;
  std::vector<std::tuple<int, cudaEvent_t, cudaEvent_t, int>> events;  // phase, start, end, kernels
  std::vector<cudaEvent_t> eventPool;
  ladds_phase_times times{};
  cudaEvent_t callStart = nullptr, callEnd = nullptr;
  std::map<std::tuple<int, int, int, size_t, size_t>, cudaGraphExec_t> graphs;
  std::string err;
  double *homeX = nullptr;  // x array of the buffer that was current at allocation
  ladds_object *dObj = nullptr;  // staging of ladds_gpu_functor_pairs (2 x objCap)
  size_t objCap = 0;
  int evalBlocks = 592;     // grid of the candidate-evaluation kernel (4 per SM)
  float cutF = 0.f;         // binary32 pre-filter radius: cutoff * (1 + nearRel), rounded up
  int chunkSteps = kMaxEphSteps;  // iterations per ephemeris chunk / captured graph (autotuned)
  uint32_t *denseCells = nullptr, *denseCount = nullptr;  // dense bin of the pair scan (cells >= kDenseCell)
  uint32_t *denseChunk = nullptr, *denseChunkB = nullptr;  // chunk index of each dense-bin entry
  uint32_t haloStart = 0xffffffffu;  // objects with slot >= haloStart: pair-scan targets only
  uint32_t denseCap = 0;
  // second set of the sort results: the sort of a step writes one set while the
  // pair scan of the previous step still reads the other
  uint32_t *rowStartB = nullptr, *keys1B = nullptr, *vals1B = nullptr, *denseCellsB = nullptr,
           *denseCountB = nullptr;
  uint16_t *cellOffB = nullptr;
  int sortParity = 0;
  struct Adjoint {          // buffers of the adjoint pair batch (ladds_gpu_adjoint_*)
    size_t nPairs = 0;
    int steps = 0, ck = 0;
    bool forwardDone = false;
    double *st = nullptr, *bc = nullptr, *aom = nullptr, *miss = nullptr, *grad = nullptr;
    double *ckpt = nullptr, *rec = nullptr, *off = nullptr;
    int *arg = nullptr;
    EphEntry *eph = nullptr;
    size_t objCap = 0, ckptCap = 0, recCap = 0, ephCap = 0;
  } adj;
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

// frees a state buffer; the slot-indexed arrays (radius, id, parent) only
// when withSlotArrays (a context's buffers share them)
void freeState(DevState &s, bool withSlotArrays) {
  void *ptrs[] = {s.x, s.y, s.z, s.vx, s.vy, s.vz, s.aom, s.bc, s.tag};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (withSlotArrays) {
    void *shared[] = {s.radius, s.id, s.parent};
    for (void *p : shared)
      if (p) cudaFree(p);
  }
  s = DevState{};
}

// allocates a state buffer; the slot-indexed arrays are taken from `shared`
// (or allocated when it has none)
cudaError_t allocState(DevState &s, size_t cap, const DevState *shared) {
  s = DevState{};
  double **d[] = {&s.x, &s.y, &s.z, &s.vx, &s.vy, &s.vz, &s.aom, &s.bc};
  for (double **p : d) {
    cudaError_t e = cudaMalloc(p, cap * sizeof(double));
    if (e != cudaSuccess) return e;
  }
  cudaError_t e = cudaMalloc(&s.tag, cap * sizeof(uint32_t));
  if (e != cudaSuccess) return e;
  if (shared) {
    s.radius = shared->radius;
    s.id = shared->id;
    s.parent = shared->parent;
    return cudaSuccess;
  }
  e = cudaMalloc(&s.radius, cap * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&s.id, cap * sizeof(uint64_t));
  if (e == cudaSuccess) e = cudaMalloc(&s.parent, cap * sizeof(uint64_t));
  return e;
}

// positions and velocities only
cudaError_t copyDynamic(const DevState &src, const DevState &dst, size_t n, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  const double *sd[] = {src.x, src.y, src.z, src.vx, src.vy, src.vz};
  double *dd[] = {dst.x, dst.y, dst.z, dst.vx, dst.vy, dst.vz};
  for (int k = 0; k < 6; ++k) {
    cudaError_t e = cudaMemcpyAsync(dd[k], sd[k], n * sizeof(double), cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// copies a state buffer (the slot-indexed arrays only when the buffers do not share them)
cudaError_t copyState(const DevState &src, const DevState &dst, size_t n, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  const double *sd[] = {src.x, src.y, src.z, src.vx, src.vy, src.vz, src.aom, src.bc};
  double *dd[] = {dst.x, dst.y, dst.z, dst.vx, dst.vy, dst.vz, dst.aom, dst.bc};
  for (int k = 0; k < 8; ++k) {
    cudaError_t e = cudaMemcpyAsync(dd[k], sd[k], n * sizeof(double), cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
  }
  cudaError_t e = cudaMemcpyAsync(dst.tag, src.tag, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st);
  if (e != cudaSuccess || src.id == dst.id) return e;
  e = cudaMemcpyAsync(dst.radius, src.radius, n * sizeof(double), cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dst.id, src.id, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dst.parent, src.parent, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, st);
  return e;
}

void dropGraphs(ladds_gpu_ctx *c) {
  for (auto &kv : c->graphs) cudaGraphExecDestroy(kv.second);
  c->graphs.clear();
}

int ensureCandCapacity(ladds_gpu_ctx *c, size_t need);

void freeBuffers(ladds_gpu_ctx *c) {
  freeState(c->cur, true);
  freeState(c->alt, false);
  freeState(c->snap, false);
  void *ptrs[] = {c->keys0, c->keys1, c->vals0, c->vals1, c->scratchA, c->scratchB, c->scratchC,
                  c->blockSums, c->posf, c->sortRec, c->scanWs, c->velf, c->keys1B, c->vals1B, c->grp};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  c->posf = nullptr;
  c->velf = nullptr;
  c->grp = nullptr;
  c->sortRec = nullptr;
  c->scanWs = nullptr;
  c->keys0 = c->keys1 = c->vals0 = c->vals1 = c->keys1B = c->vals1B = nullptr;
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
  cudaError_t e = allocState(ncur, newCap, nullptr);
  if (e == cudaSuccess) e = allocState(nalt, newCap, &ncur);
  if (e == cudaSuccess) e = allocState(nsnap, newCap, &ncur);
  if (e != cudaSuccess) {
    freeState(ncur, true);
    freeState(nalt, false);
    freeState(nsnap, false);
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
  const size_t scanBlocks = (newCap + 1 + kScanBlock - 1) / kScanBlock;
  uint32_t **u[] = {&c->keys0,    &c->keys1,    &c->vals0,  &c->vals1, &c->scratchA,
                    &c->scratchB, &c->scratchC, &c->keys1B, &c->vals1B};
  for (uint32_t **p : u) {
    if (cudaMalloc(p, (newCap + 1) * sizeof(uint32_t)) != cudaSuccess) {
      cudaGetLastError();
      return fail(c, LADDS_ERR_ALLOC, "device allocation failed (sort buffers)");
    }
  }
  // block sums of the three-level exclusive scans (objects or rows, whichever is longer)
  const size_t scanLen = std::max(newCap + 1, (size_t)c->nRows + 1);
  const size_t wsWords = 4 * (scanLen / kScanBlock + 2) + 4 * kScanBlock;
  if (cudaMalloc(&c->posf, newCap * sizeof(float4)) != cudaSuccess ||
      cudaMalloc(&c->velf, newCap * sizeof(float4)) != cudaSuccess ||
      cudaMalloc(&c->grp, newCap * sizeof(uint32_t)) != cudaSuccess ||
      cudaMalloc(&c->sortRec, newCap * sizeof(unsigned long long)) != cudaSuccess ||
      cudaMalloc(&c->scanWs, wsWords * sizeof(uint32_t)) != cudaSuccess ||
      cudaMalloc(&c->blockSums, (scanBlocks + 1) * sizeof(uint32_t)) != cudaSuccess) {
    cudaGetLastError();
    return fail(c, LADDS_ERR_ALLOC, "device allocation failed (cell-order buffers)");
  }
  for (uint32_t **p : {&c->denseCells, &c->denseCellsB, &c->denseChunk, &c->denseChunkB}) {
    if (*p) cudaFree(*p);
    *p = nullptr;
  }
  // every listed cell holds >= kDenseCell objects and adds one entry per kTileChunk of them and part of
  // its staged side (up to 2^kTilePartsLogMax parts, for cells of >= 64 * 4^kTilePartsLogMax objects)
  c->denseCap = (uint32_t)(newCap / kDenseCell + newCap / kTileChunk * (1u << kTilePartsLogMax) + 1);
  for (uint32_t **p : {&c->denseCells, &c->denseCellsB, &c->denseChunk, &c->denseChunkB}) {
    if (cudaMalloc(p, (size_t)c->denseCap * sizeof(uint32_t)) != cudaSuccess) {
      cudaGetLastError();
      for (uint32_t **q : {&c->denseCells, &c->denseCellsB, &c->denseChunk, &c->denseChunkB}) {
        if (*q) cudaFree(*q);
        *q = nullptr;
      }
      c->denseCap = 0;
      return fail(c, LADDS_ERR_ALLOC, "device allocation failed (dense-cell list)");
    }
  }
  c->cap = newCap;
  c->orderValid = false;
  dropGraphs(c);
  // candidates that pass the closest-approach screen: a few per thousand objects at LEO
  // densities; the buffer grows on overflow
  return ensureCandCapacity(c, std::max<size_t>(newCap / 8, (size_t)1 << 16));
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

int ensureCandCapacity(ladds_gpu_ctx *c, size_t need) {
  if (need <= c->candCap) return LADDS_OK;
  size_t newCap = std::max<size_t>(need + need / 2, 1);
  uint2 *p = nullptr;  // the screened and the spilled list, newCap entries each
  if (cudaMalloc(&p, 2 * newCap * sizeof(uint2)) != cudaSuccess) {
    cudaGetLastError();
    return fail(c, LADDS_ERR_ALLOC, "device allocation failed (candidate buffer)");
  }
  if (c->dCand) cudaFree(c->dCand);
  c->dCand = p;
  c->candCap = newCap;
  dropGraphs(c);
  return LADDS_OK;
}

// After a scan call: grows the record / candidate buffers that overflowed.
// *overflow tells whether the call has to be re-run.
int growIfOverflowed(ladds_gpu_ctx *c, unsigned long long *records, bool *overflow) {
  unsigned long long words[2] = {0, 0};  // record count, largest candidate count (adjacent)
  CK(cudaMemcpy(words, c->dCount, sizeof(words), cudaMemcpyDeviceToHost));
  const unsigned long long cnt = words[0], need = words[1];
  *records = cnt;
  *overflow = cnt > c->pairCap || need > c->candCap;
  if (cnt > c->pairCap) {
    const int rc = ensurePairCapacity(c, (size_t)cnt);
    if (rc) return rc;
  }
  if (need > c->candCap) {
    const int rc = ensureCandCapacity(c, (size_t)need);
    if (rc) return rc;
  }
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

// CUDA events around one phase on the stream that runs it (profiling only)
struct PhaseScope {
  ladds_gpu_ctx *c;
  int phase;
  cudaStream_t s;
  int kernels;
  cudaEvent_t a = nullptr;
  PhaseScope(ladds_gpu_ctx *c_, int ph, cudaStream_t s_, int kernels_ = 1)
      : c(c_), phase(ph), s(s_), kernels(kernels_) {
    if (c->profiling) {
      a = takeEvent(c);
      cudaEventRecord(a, s);
    }
  }
  ~PhaseScope() {
    if (c->profiling) {
      cudaEvent_t b = takeEvent(c);
      cudaEventRecord(b, s);
      c->events.emplace_back(phase, a, b, kernels);
    }
  }
};

void collectTimes(ladds_gpu_ctx *c) {
  for (auto &t : c->events) {
    float ms = 0;
    cudaEventElapsedTime(&ms, std::get<1>(t), std::get<2>(t));
    ladds_phase_times &T = c->times;
    const int k = std::get<3>(t);
    switch (std::get<0>(t)) {
      case kPhProp:
        T.propagateMs += ms;
        T.propagateLaunches += k;
        break;
      case kPhBucket:
        T.bucketMs += ms;
        T.bucketLaunches += k;
        break;
      case kPhRowsort:
        T.rowsortMs += ms;
        T.rowsortLaunches += k;
        break;
      case kPhPermute:
        T.permuteMs += ms;
        T.permuteLaunches += k;
        break;
      case kPhCandidates:
        T.candidatesMs += ms;
        T.candidatesLaunches += k;
        break;
      default:
        T.evaluateMs += ms;
        T.evaluateLaunches += k;
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
  k_ephemeris_dev<<<blocksFor(threads, 128), 128, 0, c->st>>>(c->dEph, nSteps, c->dIter, c->dIterBase,
                                                                c->cfg.startTime, c->cfg.deltaT, c->pc.hc1,
                                                                c->pc.hc2, c->cfg.epochJD, c->theta0);
  return cudaMemcpyToSymbolAsync(c_eph, c->dEph, (size_t)threads * sizeof(EphEntry), 0, cudaMemcpyDeviceToDevice,
                                 c->st);
}

// the bulk copies of k_propagate_staged need 16-byte aligned arrays
bool stageable(const DevState &s) {
  const void *p[] = {s.x, s.y, s.z, s.vx, s.vy, s.vz, s.aom, s.bc, s.tag};
  for (const void *q : p)
    if (reinterpret_cast<uintptr_t>(q) & 15u) return false;
  return true;
}

// the propagation kernel over objects [0, n) of s on the main stream; with
// keys, their cell keys and row arrivals go to keyOut / arrOut (indexed as s)
void launchPropagate(ladds_gpu_ctx *c, const DevState &s, int n, int nSteps, int ephBase, bool keys,
                     uint32_t *keyOut, uint32_t *arrOut) {
  const int b = c->cfg.propagateBlock > 0 ? c->cfg.propagateBlock : 256;
  const int g = blocksFor((size_t)n, b);
  uint32_t *rc = c->rowCounts;
  if (keys && stageable(s)) {  // the per-scan propagation: persistent grid, state staged by bulk copies
    // two CTAs per SM: alone the kernel is faster with four, but it runs beside
    // the previous iteration's pair scan, which the other slots then serve
    const int sg = std::max(1, std::min(blocksFor((size_t)n, kStageObjects), c->evalBlocks / 2));
    if (c->cfg.precision == LADDS_PRECISION_SPLIT)
      k_propagate_staged<true><<<sg, kStageObjects, 0, c->st>>>(s, n, nSteps, ephBase, c->pc, c->grid, keyOut, rc,
                                                                arrOut, c->dStatus);
    else
      k_propagate_staged<false><<<sg, kStageObjects, 0, c->st>>>(s, n, nSteps, ephBase, c->pc, c->grid, keyOut, rc,
                                                                 arrOut, c->dStatus);
    return;
  }
  if (c->cfg.precision == LADDS_PRECISION_SPLIT) {
    if (keys)
      k_propagate<true, true><<<g, b, 0, c->st>>>(s, n, nSteps, ephBase, c->pc, c->grid, keyOut, rc, arrOut,
                                                  c->dStatus);
    else
      k_propagate<true, false><<<g, b, 0, c->st>>>(s, n, nSteps, ephBase, c->pc, c->grid, nullptr, nullptr, nullptr,
                                                   c->dStatus);
  } else {
    if (keys)
      k_propagate<false, true><<<g, b, 0, c->st>>>(s, n, nSteps, ephBase, c->pc, c->grid, keyOut, rc, arrOut,
                                                   c->dStatus);
    else
      k_propagate<false, false><<<g, b, 0, c->st>>>(s, n, nSteps, ephBase, c->pc, c->grid, nullptr, nullptr,
                                                    nullptr, c->dStatus);
  }
}

// nSteps steps whose stage ephemerides are c_eph[ephBase ...]
void enqueuePropagate(ladds_gpu_ctx *c, int nSteps, bool keys, int ephBase) {
  if (c->n == 0) {
    k_advance<<<1, 32, 0, c->st>>>(c->dIter, nSteps);
    return;
  }
  // with keys: the row counts of the coming sort are accumulated by the kernel
  if (keys) cudaMemsetAsync(c->rowCounts, 0, ((size_t)c->nRows + 1) * sizeof(uint32_t), c->st);
  PhaseScope ps(c, kPhProp, c->st, 2);  // propagation + iteration counter
  launchPropagate(c, c->cur, (int)c->n, nSteps, ephBase, keys, c->keys0, c->scratchC);
  k_advance<<<1, 32, 0, c->st>>>(c->dIter, nSteps);
}

// kernels launched by enqueueExclusiveScan for `count` values
constexpr bool kScanFoldSums = true;  // two passes up to kScanBlock^2 values (else three)

int exclusiveScanKernels(size_t count) {
  const int nb1 = blocksFor(count, kScanBlock);
  if (nb1 == 1) return 1;
  if (kScanFoldSums && nb1 <= kScanBlock) return 2;
  return blocksFor((size_t)nb1, kScanBlock) > 1 ? 5 : 3;
}

// exclusive scan of `count` u32 values (1024-wide block scans; up to 2^20
// values: block scans, then each block adds the sum of the blocks before it;
// beyond: three levels, count <= 2^30); block sums live in c->scanWs
void enqueueExclusiveScan(ladds_gpu_ctx *c, const uint32_t *in, size_t count, uint32_t *out) {
  const int nb1 = blocksFor(count, kScanBlock);
  uint32_t *s1 = c->scanWs, *s1x = s1 + nb1 + 1;
  k_scan_blocks<<<nb1, kScanBlock, 0, c->st>>>(in, (int)count, out, s1);
  if (nb1 == 1) return;
  if (kScanFoldSums && nb1 <= kScanBlock) {
    k_scan_add_prefix<<<nb1, kScanBlock, 0, c->st>>>(out, (int)count, s1);
    return;
  }
  const int nb2 = blocksFor((size_t)nb1, kScanBlock);
  uint32_t *s2 = s1x + nb1 + 1;
  k_scan_blocks<<<nb2, kScanBlock, 0, c->st>>>(s1, nb1, s1x, s2);
  if (nb2 > 1) {
    uint32_t *s2x = s2 + nb2 + 1, *s3 = s2x + nb2 + 1;
    k_scan_blocks<<<1, kScanBlock, 0, c->st>>>(s2, nb2, s2x, s3);
    k_scan_add<<<nb2, kScanBlock, 0, c->st>>>(s1x, nb1, s2x);
  }
  k_scan_add<<<nb1, kScanBlock, 0, c->st>>>(out, (int)count, s1x);
}

// the dense bin of the pair scan: on with the counting row sort and the cell tables
DenseBin denseBin(const ladds_gpu_ctx *c) {
  const bool on = c->cellOff && c->denseCells && (uint32_t)c->grid.n[0] <= (uint32_t)kRowCountMaxNx &&
                  c->grid.reach <= 3;  // k_pair_tiles: one lane per half-shell row (<= 25 rows)
  return DenseBin{on ? c->denseCells : nullptr, c->denseCount, c->denseCap, kDenseCell, c->denseChunk};
}

// the sort writes the result set that the previous pair scan does not read
void swapSortSets(ladds_gpu_ctx *c) {
  std::swap(c->rowStart, c->rowStartB);
  std::swap(c->keys1, c->keys1B);
  std::swap(c->vals1, c->vals1B);
  std::swap(c->cellOff, c->cellOffB);
  std::swap(c->denseCells, c->denseCellsB);
  std::swap(c->denseChunk, c->denseChunkB);
  std::swap(c->denseCount, c->denseCountB);
  c->sortParity ^= 1;
}

// keys0 holds the keys of c->cur in current order, rowCounts their row counts
// and scratchC their arrival indices (k_propagate<*, true> or k_cell_keys) ->
// sortedKeys (keys1), perm (vals1) and the row-start table; order = sort by
// (cell key, slot)
void enqueueSort(ladds_gpu_ctx *c) {
  swapSortSets(c);
  const int n = (int)c->n;
  const uint32_t nx = (uint32_t)c->grid.n[0], nRows = c->nRows;
  {
    PhaseScope ps(c, kPhBucket, c->st, 1 + exclusiveScanKernels((size_t)nRows + 1));
    cudaMemsetAsync(c->longCount, 0, sizeof(uint32_t), c->st);
    cudaMemsetAsync(c->denseCount, 0, sizeof(uint32_t), c->st);
    enqueueExclusiveScan(c, c->rowCounts, (size_t)nRows + 1, c->rowStart);
    k_bucket_place<<<blocksFor(c->n, kBucketThreads), kBucketThreads, 0, c->st>>>(
        c->keys0, c->scratchC, c->cur.tag, n, nx, c->rowStart, c->sortRec, c->vals0, c->dStatus);
  }
  PhaseScope ps(c, kPhRowsort, c->st, 2);
  const DenseBin dense = denseBin(c);
  if (nx <= (uint32_t)kRowCountMaxNx) {  // counting sort inside the rows
    // one resident wave (8 CTAs of 4 warps per SM by shared memory); each warp pipelines its rows
    const int rowBlocks = std::min(blocksFor((size_t)nRows * 32, kRowSortThreads), 2 * c->evalBlocks);
    k_bucket_sort_rows<<<rowBlocks, kRowSortThreads, rowSortSmem(nx), c->st>>>(
        c->rowStart, nRows, nx, c->sortRec, c->vals0, c->keys1, c->vals1, c->longRows, c->longCount, c->cellOff,
        dense);
  } else {
    const int smallBlocks = std::min(blocksFor((size_t)nRows * 32, kBucketThreads), 16 * c->evalBlocks);
    k_bucket_sort_small<<<smallBlocks, kBucketThreads, 0, c->st>>>(
        c->rowStart, nRows, nx, c->sortRec, c->vals0, c->keys1, c->vals1, c->longRows, c->longCount, c->cellOff);
  }
  k_bucket_sort_large<<<c->evalBlocks / 2, kBucketThreads, kLargeRow * 12, c->st>>>(
      c->rowStart, nx, c->sortRec, c->vals0, c->keys1, c->vals1, c->longRows, c->longCount, c->cellOff, dense);
  c->sortedKeys = c->keys1;
  c->perm = c->vals1;
}

// after the gather (enqueueCells) alt holds the state as the scan sees it, perm maps into it
inline ScanPack scanPack(ladds_gpu_ctx *c) {
  return ScanPack{c->posf, c->velf, c->alt, c->perm, c->anyParent ? c->grp : nullptr};
}

// gathers the state into cell order (so that the next propagation, key pass and
// gather read nearly sequentially: objects move about one cell per step) and
// writes the packed scan copies
void enqueueCells(ladds_gpu_ctx *c) {
  PhaseScope ps(c, kPhPermute, c->st);
  k_permute<<<blocksFor(c->n, 256), 256, 0, c->st>>>(c->cur, c->alt, c->perm, (int)c->n, scanPack(c),
                                                      c->dStatus);
  std::swap(c->cur, c->alt);
}

// binary32 pre-filter radius of a cutoff: cutoff * (1 + nearRel), rounded up
inline float prefilterRadius(double cutoff, double nearRel) {
  return (float)(cutoff * (1.0 + nearRel) * (1.0 + 1e-6));
}

// candidates + evaluation on stream s; records carry *iterPtr + iterOffset
void enqueueScanWith(ladds_gpu_ctx *c, cudaStream_t s, const ScanConsts &scIn, float cutF, const int64_t *iterPtr,
                     int64_t iterOffset) {
  const ScanConsts sc = screenConsts(scIn);
  const DenseBin dense = denseBin(c);
  {
    PhaseScope ps(c, kPhCandidates, s, dense.cells ? 2 : 1);
    // the two list lengths and the dense bin's next-entry counter
    cudaMemsetAsync(c->dCandCount, 0, 3 * sizeof(unsigned long long), s);
    const CandSink out{sc,       c->posf,     c->velf,      c->dCand, c->dCandCount, (unsigned long long)c->candCap,
                       c->haloStart, c->anyParent ? c->grp : nullptr};
    const bool buffer = c->cfg.scanScreen == LADDS_SCREEN_BUFFER;
    // the largest separation a record or a near-band flag can have, with room for rounding
    const double reach = std::sqrt(sc.cutoffSq) * (1.0 + sc.nearRel) * (1.0 + 1e-6);
    const uint32_t denseMin = dense.cells ? dense.minCount : 0xffffffffu;
    const int form = c->cfg.walkForm != LADDS_WALK_AUTO
                         ? c->cfg.walkForm
                         : (!buffer && c->grid.reach == 1 ? LADDS_WALK_GROUPED : LADDS_WALK_ROWS);
    if (form == LADDS_WALK_ROWS) {
      (buffer ? k_pair_rows<LADDS_SCREEN_BUFFER> : k_pair_rows<LADDS_SCREEN_LISTS>)<<<blocksFor(c->n, kScanCta),
                                                                                       kScanCta, 0, s>>>(
          c->cur.tag, c->posf, (int)c->n, c->sortedKeys, c->rowStart, c->cellOff, c->grid, cutF, reach * reach,
          denseMin, c->denseCount, out);
    } else {
      HalfShellRows rows;
      buildHalfShellRows(rows, c->grid.reach, c->grid.cellSize, reach * reach);
      const bool r1 = c->grid.reach == 1 && rows.n == 5;  // the five reach-1 rows, all of half-width 1
      auto walk = buffer ? (r1 ? k_pair_candidates<LADDS_SCREEN_BUFFER, true>
                               : k_pair_candidates<LADDS_SCREEN_BUFFER, false>)
                         : (r1 ? k_pair_candidates<LADDS_SCREEN_LISTS, true>
                               : k_pair_candidates<LADDS_SCREEN_LISTS, false>);
      walk<<<blocksFor(c->n, kScanCta), kScanCta, 0, s>>>(c->cur.tag, c->posf, (int)c->n, c->sortedKeys,
                                                          c->rowStart, c->cellOff, c->grid, cutF, reach * reach,
                                                          denseMin, c->denseCount, rows, out);
    }
    if (dense.cells)  // the dense bin: grid-stride over the listed cells (count read on the device)
      (buffer ? k_pair_tiles<LADDS_SCREEN_BUFFER>
              : k_pair_tiles<LADDS_SCREEN_LISTS>)<<<4 * c->evalBlocks, kScanCta, 0, s>>>(
          dense.cells, dense.chunk, dense.count, dense.cap, c->cur.tag, c->posf, c->sortedKeys, c->rowStart,
          c->cellOff, c->grid, cutF, reach * reach, out);
  }
  PhaseScope ps(c, kPhEvaluate, s);
  const int b = c->cfg.scanBlock > 0 ? c->cfg.scanBlock : 256;
  // grid-stride over both candidate lists (their lengths are only known on the device): one resident wave
  const int evalGrid = std::max(1, std::min(blocksFor(2 * c->candCap, b), c->evalBlocks * 256 / b));
  k_pair_eval<<<evalGrid, b, 0, s>>>(scanPack(c), c->dCand, c->dCandCount, (unsigned long long)c->candCap,
                                     c->dCandNeed, sc, iterPtr, iterOffset, c->dPairs, c->dCount,
                                     (unsigned long long)c->pairCap);
}

// one iteration; its stage ephemerides are entries 3*slot.. of the chunk table in c_eph
// `len` iterations starting at iteration itStart (len <= kMaxEphSteps): one
// ephemeris kernel + one constant-memory copy for the whole chunk.  The pair
// scan of iteration i (candidates + evaluation) runs on the second stream,
// concurrently with the propagation and the sort of the next scanned
// iteration: the scan reads the packed cell-order copies, the pre-gather state,
// the tags and one set of sort results; the propagation writes none of them and
// the sort writes the other set.  The next gather, which overwrites the packed
// copies and the pre-gather state, waits for the scan.  Records carry the
// chunk's first iteration (stored by the ephemeris kernel) + i.
void enqueueChunk(ladds_gpu_ctx *c, int64_t itStart, int len, int k) {
  enqueueEphemeris(c, len);
  const bool overlap = !c->profiling;
  bool pending = false;  // a scan on the second stream that the main stream has not joined
  for (int i = 0; i < len; ++i) {
    const bool scan = ((itStart + i) % k) == 0 && c->n;
    enqueuePropagate(c, 1, scan, 3 * i);
    if (!scan) continue;
    enqueueSort(c);
    if (pending) {
      cudaStreamWaitEvent(c->st, c->evScan, 0);
      pending = false;
    }
    enqueueCells(c);
    ScanConsts sc = c->sc;
    sc.dt = c->cfg.deltaT * (double)k;
    if (overlap) {
      cudaEventRecord(c->evCells, c->st);
      cudaStreamWaitEvent(c->st2, c->evCells, 0);
      enqueueScanWith(c, c->st2, sc, c->cutF, c->dIterBase, i);
      cudaEventRecord(c->evScan, c->st2);
      pending = true;
    } else {
      enqueueScanWith(c, c->st, sc, c->cutF, c->dIterBase, i);
    }
  }
  if (pending) cudaStreamWaitEvent(c->st, c->evScan, 0);
}

// host-side effect of replaying a captured chunk: the buffer swaps of its scans
void replaySwaps(ladds_gpu_ctx *c, int64_t itStart, int len, int k) {
  int scans = 0;
  for (int i = 0; i < len; ++i) scans += ((itStart + i) % k) == 0;
  if (!scans || !c->n) return;
  if (scans % 2 == 1) {
    std::swap(c->cur, c->alt);
    swapSortSets(c);
  }
  c->sortedKeys = c->keys1;
  c->perm = c->vals1;
}

int syncAndStatus(ladds_gpu_ctx *c) {
  CK(cudaStreamSynchronize(c->st));
  CK(cudaGetLastError());
  unsigned status = 0;
  CK(cudaMemcpy(&status, c->dStatus, sizeof(unsigned), cudaMemcpyDeviceToHost));
  if (status) CK(cudaMemset(c->dStatus, 0, sizeof(unsigned)));
  if (status & 4u) return fail(c, LADDS_ERR_DEVICE_CHECK, "a device-side index check failed (sort / gather)");
  if (status & 8u) return fail(c, LADDS_ERR_DEVICE_CHECK, "a bounded device wait ran out (staged propagation)");
  if (status & 1u) return fail(c, LADDS_ERR_NONFINITE, "a position or velocity became NaN/Inf during propagation");
  return LADDS_OK;
}

// syncAndStatus + growIfOverflowed with one read of the three words after the sync
int syncStatusAndGrow(ladds_gpu_ctx *c, unsigned long long *records, bool *overflow) {
  CK(cudaStreamSynchronize(c->st));
  CK(cudaGetLastError());
  unsigned long long w[3] = {0, 0, 0};  // record count, largest candidate count, status
  CK(cudaMemcpy(w, c->dCount, sizeof(w), cudaMemcpyDeviceToHost));
  const unsigned status = (unsigned)(w[2] & 0xffffffffull);
  if (status) CK(cudaMemset(c->dStatus, 0, sizeof(unsigned)));
  if (status & 4u) return fail(c, LADDS_ERR_DEVICE_CHECK, "a device-side index check failed (sort / gather)");
  if (status & 8u) return fail(c, LADDS_ERR_DEVICE_CHECK, "a bounded device wait ran out (staged propagation)");
  if (status & 1u) return fail(c, LADDS_ERR_NONFINITE, "a position or velocity became NaN/Inf during propagation");
  *records = w[0];
  *overflow = w[0] > c->pairCap || w[1] > c->candCap;
  if (w[0] > c->pairCap) {
    const int rc = ensurePairCapacity(c, (size_t)w[0]);
    if (rc) return rc;
  }
  if (w[1] > c->candCap) {
    const int rc = ensureCandCapacity(c, (size_t)w[1]);
    if (rc) return rc;
  }
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
  for (size_t i = 0; i < n && parentId && !c->anyParent; ++i) c->anyParent = parentId[i] != UINT64_MAX;
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

void freeGridBuffers(ladds_gpu_ctx *c) {
  void *ptrs[] = {c->rowStart, c->rowStartB, c->rowCounts, c->longRows, c->cellOff, c->cellOffB};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  c->rowStart = c->rowStartB = c->rowCounts = c->longRows = nullptr;
  c->cellOff = c->cellOffB = nullptr;
}

// row tables of c->grid; the two cell-offset tables when each fits 512 MiB (250^3 cells: 31 MB)
int allocGridBuffers(ladds_gpu_ctx *c) {
  if (cudaMalloc(&c->rowStart, ((size_t)c->nRows + 1) * sizeof(uint32_t)) != cudaSuccess ||
      cudaMalloc(&c->rowStartB, ((size_t)c->nRows + 1) * sizeof(uint32_t)) != cudaSuccess ||
      cudaMalloc(&c->rowCounts, 2 * ((size_t)c->nRows + 1) * sizeof(uint32_t)) != cudaSuccess ||
      cudaMalloc(&c->longRows, ((size_t)c->nRows + 1) * sizeof(uint32_t)) != cudaSuccess) {
    cudaGetLastError();
    freeGridBuffers(c);
    return fail(c, LADDS_ERR_ALLOC, "device allocation of the cell-row tables failed");
  }
  const size_t cellOffBytes = (size_t)c->nRows * cellOffPitch((uint32_t)c->grid.n[0]) * sizeof(uint16_t);
  if (cellOffBytes <= ((size_t)1 << 29) && (cudaMalloc(&c->cellOff, cellOffBytes) != cudaSuccess ||
                                               cudaMalloc(&c->cellOffB, cellOffBytes) != cudaSuccess)) {
    cudaGetLastError();
    if (c->cellOff) cudaFree(c->cellOff);
    c->cellOff = c->cellOffB = nullptr;  // the scan then searches the sorted keys
  }
  return LADDS_OK;
}

constexpr size_t kHostCopyBlock = (size_t)1 << 17;  // doubles per task of the staging copies

bool isPinned(const void *p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// dst[a][lo, lo + len) = src[a][lo, lo + len) for the arrays with use[a], on all host threads
void hostCopy(double *const dst[6], const double *const src[6], const bool use[6], size_t lo, size_t len) {
  const long per = (long)((len + kHostCopyBlock - 1) / kHostCopyBlock);
#pragma omp parallel for schedule(static)
  for (long t = 0; t < 6 * per; ++t) {
    const int a = (int)(t / per);
    if (!use[a]) continue;
    const size_t b = lo + (size_t)(t % per) * kHostCopyBlock, e = std::min(b + kHostCopyBlock, lo + len);
    std::memcpy(dst[a] + b, src[a] + b, (e - b) * sizeof(double));
  }
}

// dst[0, n) = src[0, n) on all host threads
void hostCopyOne(double *dst, const double *src, size_t n) {
  const double *const s6[6] = {src, nullptr, nullptr, nullptr, nullptr, nullptr};
  double *const d6[6] = {dst, nullptr, nullptr, nullptr, nullptr, nullptr};
  const bool use[6] = {true, false, false, false, false, false};
  hostCopy(d6, s6, use, 0, n);
}

// the context's pinned staging buffer for pageable host arrays: 12 arrays of
// at least n doubles (six in, six out); false if no pinned memory is to be had
// (the CUDA driver then stages the copies itself)
bool ensurePinStage(ladds_gpu_ctx *c, size_t n) {
  if (c->pinStage && c->pinCap >= n) return true;
  if (c->pinStage) cudaFreeHost(c->pinStage);
  c->pinStage = nullptr;
  c->pinCap = 0;
  if (cudaHostAlloc(&c->pinStage, 12 * n * sizeof(double), cudaHostAllocDefault) != cudaSuccess) {
    cudaGetLastError();
    c->pinStage = nullptr;
    return false;
  }
  c->pinCap = n;
  return true;
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
  f->scanBlock = 256;
  f->useGraphs = 1;
  f->pairCapacity = 0;
  f->scanScreen = LADDS_SCREEN_LISTS;
  f->walkForm = LADDS_WALK_AUTO;
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
      f->scanBlock > 256 || (f->scanBlock % 32) ||
      (f->scanScreen != LADDS_SCREEN_LISTS && f->scanScreen != LADDS_SCREEN_BUFFER) ||
      (f->walkForm != LADDS_WALK_AUTO && f->walkForm != LADDS_WALK_GROUPED && f->walkForm != LADDS_WALK_ROWS))
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
  c->cutF = (float)(f->cutoff * (1.0 + f->nearThresholdRel) * (1.0 + 1e-6));
  c->theta0 = gmstIAU1982(f->epochJD);
  if (cudaSetDevice(c->dev) != cudaSuccess || cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess ||
      allocGridBuffers(c) != LADDS_OK || cudaMalloc(&c->longCount, sizeof(uint32_t)) != cudaSuccess ||
      cudaMalloc(&c->denseCount, sizeof(uint32_t)) != cudaSuccess ||
      cudaMalloc(&c->denseCountB, sizeof(uint32_t)) != cudaSuccess ||
      cudaMalloc(&c->dCount, 3 * sizeof(unsigned long long)) != cudaSuccess ||
      cudaMalloc(&c->dCandCount, 3 * sizeof(unsigned long long)) != cudaSuccess ||
      cudaMalloc(&c->dEph, 3 * kMaxEphSteps * sizeof(EphEntry)) != cudaSuccess ||
      cudaMalloc(&c->dIter, 2 * sizeof(int64_t)) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->st2, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->st3, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    ladds_gpu_destroy(c);
    return LADDS_ERR_ALLOC;
  }
  c->dIterBase = c->dIter + 1;
  // record count, largest candidate count and status words side by side: one read after a step
  c->dCandNeed = c->dCount + 1;
  c->dStatus = reinterpret_cast<unsigned *>(c->dCount + 2);
  cudaMemset(c->dCount, 0, 3 * sizeof(unsigned long long));
  cudaMemset(c->dIter, 0, 2 * sizeof(int64_t));
  cudaEventCreate(&c->callStart);
  cudaEventCreate(&c->callEnd);
  cudaEventCreateWithFlags(&c->evCells, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&c->evScan, cudaEventDisableTiming);
  for (auto &e : c->evXfer) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
  for (auto &e : c->evPipe) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
  cudaMemset(c->dCandCount, 0, 3 * sizeof(unsigned long long));
  cudaMemset(c->dCandNeed, 0, sizeof(unsigned long long));
  c->evalBlocks = 4 * std::max(prop.multiProcessorCount, 1);
  // The reach-1 list walk runs beside the propagation and the sort of the next
  // iteration; at its 40 registers twelve of its CTAs fit an SM, and the extra
  // resident warps slow the iteration beside them more than they speed the
  // walk.  A shared-memory carveout of 132 KB (57 % of 228 KB) holds it at ten
  // CTAs per SM: 10 x (12 KB + 1 KB reserved).
  if (cudaFuncSetAttribute(k_pair_candidates<LADDS_SCREEN_LISTS, true>, cudaFuncAttributePreferredSharedMemoryCarveout,
                           57) != cudaSuccess)
    cudaGetLastError();  // a preference only: without it the walk runs with more CTAs per SM
  rc = ensurePairCapacity(c, f->pairCapacity ? (size_t)f->pairCapacity : (size_t)1 << 16);
  if (!rc) rc = ensureCandCapacity(c, (size_t)1 << 16);
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
  freeGridBuffers(c);
  void *ptrs[] = {c->longCount, c->denseCount, c->denseCells, c->denseCountB, c->denseCellsB, c->dCount,
                  c->denseChunk, c->denseChunkB, c->dEph,
                  c->dIter, c->dPairs, c->dCand, c->dCandCount, c->dObj,
                  c->adj.st, c->adj.bc, c->adj.aom, c->adj.miss, c->adj.grad, c->adj.ckpt, c->adj.rec,
                  c->adj.off, c->adj.arg, c->adj.eph};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  for (auto &t : c->events) {
    cudaEventDestroy(std::get<1>(t));
    cudaEventDestroy(std::get<2>(t));
  }
  for (auto e : c->eventPool) cudaEventDestroy(e);
  if (c->callStart) cudaEventDestroy(c->callStart);
  if (c->callEnd) cudaEventDestroy(c->callEnd);
  if (c->evCells) cudaEventDestroy(c->evCells);
  if (c->evScan) cudaEventDestroy(c->evScan);
  for (auto e : c->evXfer)
    if (e) cudaEventDestroy(e);
  for (auto e : c->evPipe)
    if (e) cudaEventDestroy(e);
  if (c->pinStage) cudaFreeHost(c->pinStage);
  if (c->st3) cudaStreamDestroy(c->st3);
  if (c->st2) cudaStreamDestroy(c->st2);
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
  c->anyParent = false;
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

int ladds_gpu_reserve(ladds_gpu_ctx *c, size_t capacity) {
  if (!c) return LADDS_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g_deviceMutex[c->dev & 63]);
  if (capacity <= c->cap) return LADDS_OK;
  CK(cudaSetDevice(c->dev));
  return ensureCapacity(c, capacity);
}

int ladds_gpu_checked_insert(ladds_gpu_ctx *c, size_t n, const double *x, const double *y, const double *z,
                             const double *vx, const double *vy, const double *vz, const double *radius,
                             const double *aom, const double *bcInv, const uint64_t *id, const uint64_t *parentId,
                             const int8_t *activity, double constellationCutoff, uint8_t *delayed,
                             size_t *nInserted) {
  if (!c || (n && (!x || !y || !z || !id || !delayed)) || !(constellationCutoff >= 0.0))
    return fail(c, LADDS_ERR_INVALID_ARG, "checked_insert: bad argument");
  if (nInserted) *nInserted = 0;
  if (!n) return LADDS_OK;
  const double cc = constellationCutoff, c2 = cc * cc;
  std::vector<uint8_t> blocked(n, 0);
  {
    std::lock_guard<std::mutex> lk(g_deviceMutex[c->dev & 63]);
    CK(cudaSetDevice(c->dev));
    if (c->n) {
      double *dp = nullptr;
      uint8_t *db = nullptr;
      if (cudaMalloc(&dp, 3 * n * sizeof(double)) != cudaSuccess || cudaMalloc(&db, n) != cudaSuccess) {
        cudaGetLastError();
        if (dp) cudaFree(dp);
        return fail(c, LADDS_ERR_ALLOC, "checked_insert: staging allocation failed");
      }
      cudaError_t e = cudaMemcpyAsync(dp, x, n * sizeof(double), cudaMemcpyHostToDevice, c->st);
      if (e == cudaSuccess) e = cudaMemcpyAsync(dp + n, y, n * sizeof(double), cudaMemcpyHostToDevice, c->st);
      if (e == cudaSuccess) e = cudaMemcpyAsync(dp + 2 * n, z, n * sizeof(double), cudaMemcpyHostToDevice, c->st);
      if (e == cudaSuccess) {
        k_insert_blocked<<<blocksFor(n * 32, 128), 128, 0, c->st>>>(c->cur, (int)c->n, dp, dp + n, dp + 2 * n,
                                                                     (int)n, cc, c2, db);
        e = cudaGetLastError();
      }
      if (e == cudaSuccess) e = cudaMemcpyAsync(blocked.data(), db, n, cudaMemcpyDeviceToHost, c->st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
      cudaFree(dp);
      cudaFree(db);
      if (e != cudaSuccess) return fail(c, LADDS_ERR_CUDA, std::string("checked_insert: ") + cudaGetErrorString(e));
    }
  }
  // satellites of the batch, in order, against the ones accepted before them
  std::vector<size_t> acc;
  for (size_t i = 0; i < n; ++i) {
    bool hit = blocked[i] != 0;
    const double p[3] = {x[i], y[i], z[i]};
    for (size_t q = 0; q < acc.size() && !hit; ++q) {
      const double o[3] = {x[acc[q]], y[acc[q]], z[acc[q]]};
      hit = insertBlocks(p, o, cc, c2);
    }
    delayed[i] = hit ? 1 : 0;
    if (!hit) acc.push_back(i);
  }
  if (acc.empty()) return LADDS_OK;
  const size_t m = acc.size();
  std::vector<double> d[9];
  const double *src[9] = {x, y, z, vx, vy, vz, radius, aom, bcInv};
  for (int k = 0; k < 9; ++k) {
    d[k].resize(m);
    for (size_t q = 0; q < m; ++q) d[k][q] = src[k] ? src[k][acc[q]] : 0.0;
  }
  std::vector<uint64_t> ids(m), parents(m);
  std::vector<int8_t> acts(m);
  for (size_t q = 0; q < m; ++q) {
    ids[q] = id[acc[q]];
    parents[q] = parentId ? parentId[acc[q]] : UINT64_MAX;
    acts[q] = activity ? activity[acc[q]] : (int8_t)LADDS_PASSIVE;
  }
  const int rc = ladds_gpu_append(c, m, d[0].data(), d[1].data(), d[2].data(), d[3].data(), d[4].data(),
                                  d[5].data(), d[6].data(), d[7].data(), d[8].data(), ids.data(), parents.data(),
                                  acts.data());
  if (!rc && nInserted) *nInserted = m;
  return rc;
}

int ladds_gpu_get_objects(ladds_gpu_ctx *c, const uint32_t *slots, size_t m, ladds_state_record *out) {
  if (!c || (m && (!slots || !out))) return fail(c, LADDS_ERR_INVALID_ARG, "get_objects: bad argument");
  if (!m) return LADDS_OK;
  std::vector<uint32_t> want(slots, slots + m);
  std::sort(want.begin(), want.end());
  want.erase(std::unique(want.begin(), want.end()), want.end());
  const int mu = (int)want.size();
  std::lock_guard<std::mutex> lk(g_deviceMutex[c->dev & 63]);
  CK(cudaSetDevice(c->dev));
  uint32_t *dWant = nullptr;
  int32_t *dPos = nullptr;
  ladds_state_record *dRec = nullptr;
  if (cudaMalloc(&dWant, mu * sizeof(uint32_t)) != cudaSuccess || cudaMalloc(&dPos, mu * sizeof(int32_t)) != cudaSuccess ||
      cudaMalloc(&dRec, mu * sizeof(ladds_state_record)) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(dWant);
    cudaFree(dPos);
    return fail(c, LADDS_ERR_ALLOC, "get_objects: staging allocation failed");
  }
  std::vector<int32_t> pos(mu, -1);
  std::vector<ladds_state_record> rec(mu);
  cudaError_t e = cudaMemcpyAsync(dWant, want.data(), mu * sizeof(uint32_t), cudaMemcpyHostToDevice, c->st);
  if (e == cudaSuccess) e = cudaMemsetAsync(dPos, 0xff, mu * sizeof(int32_t), c->st);
  if (e == cudaSuccess && c->n)
    k_find_slots<<<blocksFor(c->n, 256), 256, 0, c->st>>>(c->cur.tag, (int)c->n, dWant, mu, dPos);
  if (e == cudaSuccess) k_gather_records<<<blocksFor((size_t)mu, 128), 128, 0, c->st>>>(c->cur, dPos, mu, dRec);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(pos.data(), dPos, mu * sizeof(int32_t), cudaMemcpyDeviceToHost, c->st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(rec.data(), dRec, mu * sizeof(ladds_state_record), cudaMemcpyDeviceToHost, c->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
  cudaFree(dWant);
  cudaFree(dPos);
  cudaFree(dRec);
  if (e != cudaSuccess) return fail(c, LADDS_ERR_CUDA, std::string("get_objects: ") + cudaGetErrorString(e));
  for (size_t q = 0; q < m; ++q) {
    const size_t k = std::lower_bound(want.begin(), want.end(), slots[q]) - want.begin();
    if (pos[k] < 0) return fail(c, LADDS_ERR_INVALID_ARG, "get_objects: no object with slot " + std::to_string(slots[q]));
    out[q] = rec[k];
  }
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
  const double *src[] = {c->cur.x, c->cur.y, c->cur.z, c->cur.vx, c->cur.vy, c->cur.vz, c->cur.aom, c->cur.bc};
  double *dst[] = {x, y, z, vx, vy, vz, aom, bcInv};
  for (int k = 0; k < 8; ++k) {
    if (!dst[k]) continue;
    k_unpermute_f64<<<g, 256, 0, c->st>>>(src[k], c->cur.tag, (int)c->n, c->alt.x);
    CK(cudaMemcpyAsync(dst[k], c->alt.x, c->n * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
  }
  // radius, id and parent are slot-indexed already
  if (radius) CK(cudaMemcpyAsync(radius, c->cur.radius, c->n * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  if (id) CK(cudaMemcpyAsync(id, c->cur.id, c->n * sizeof(uint64_t), cudaMemcpyDeviceToHost, c->st));
  if (parentId)
    CK(cudaMemcpyAsync(parentId, c->cur.parent, c->n * sizeof(uint64_t), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
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
  // pageable arrays go through the context's pinned staging, copied on all host
  // threads while the previous array crosses PCIe
  bool pinned[6], staged = false;
  for (int k = 0; k < 6; ++k) {
    pinned[k] = isPinned(src[k]);
    staged |= !pinned[k];
  }
  if (staged && !ensurePinStage(c, n))
    for (bool &p : pinned) p = true;  // no pinned memory to spare: the driver stages them
  // the copies run back to back on the main stream; each array's gather into
  // cell order runs on the second stream while the next array crosses PCIe
  for (int k = 0; k < 6; ++k) {
    const double *from = src[k];
    if (!pinned[k]) {
      double *pin = c->pinStage + (size_t)k * c->pinCap;
      hostCopyOne(pin, src[k], n);
      from = pin;
    }
    CK(cudaMemcpyAsync(stage[k], from, n * sizeof(double), cudaMemcpyHostToDevice, c->st));
    CK(cudaEventRecord(c->evXfer[k], c->st));
    CK(cudaStreamWaitEvent(c->st2, c->evXfer[k], 0));
    k_permute_from_slots_f64<<<g, 256, 0, c->st2>>>(stage[k], c->cur.tag, (int)n, dst[k]);
  }
  CK(cudaStreamSynchronize(c->st2));
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
  // scatters into slot order on the second stream, all launched before the
  // first copy (a copy into pageable memory blocks the host); each array's
  // copy waits for its own scatter only
  CK(cudaEventRecord(c->evXfer[6], c->st));
  CK(cudaStreamWaitEvent(c->st2, c->evXfer[6], 0));
  for (int k = 0; k < 6; ++k) {
    if (!dst[k]) continue;
    k_unpermute_f64<<<g, 256, 0, c->st2>>>(src[k], c->cur.tag, (int)c->n, stage[k]);
    CK(cudaEventRecord(c->evXfer[k], c->st2));
  }
  // pageable arrays come back through the context's pinned staging: each
  // array leaves the pinned buffer on all host threads while the next crosses PCIe
  bool pinned[6], staged = false;
  for (int k = 0; k < 6; ++k) {
    pinned[k] = !dst[k] || isPinned(dst[k]);
    staged |= !pinned[k];
  }
  if (staged && !ensurePinStage(c, c->n))
    for (bool &p : pinned) p = true;  // no pinned memory to spare: the driver stages them
  for (int k = 0; k < 6; ++k) {
    if (!dst[k]) continue;
    CK(cudaStreamWaitEvent(c->st, c->evXfer[k], 0));
    double *to = pinned[k] ? dst[k] : c->pinStage + (size_t)(6 + k) * c->pinCap;
    CK(cudaMemcpyAsync(to, stage[k], c->n * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaEventRecord(c->evPipe[k], c->st));
  }
  for (int k = 0; k < 6; ++k) {
    if (!dst[k] || pinned[k]) continue;
    CK(cudaEventSynchronize(c->evPipe[k]));
    hostCopyOne(dst[k], c->pinStage + (size_t)(6 + k) * c->pinCap, c->n);
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
  t->totalMs = t->propagateMs + t->bucketMs + t->rowsortMs + t->permuteMs + t->candidatesMs + t->evaluateMs;
  return LADDS_OK;
}

int ladds_gpu_integrate(ladds_gpu_ctx *c, int steps) {
  if (!c || steps < 0) return LADDS_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g_deviceMutex[c->dev & 63]);
  CK(cudaSetDevice(c->dev));
  int left = steps;
  while (left > 0) {
    const int chunk = std::min(left, c->chunkSteps);
    CK(enqueueEphemeris(c, chunk));
    enqueuePropagate(c, chunk, false, 0);
    left -= chunk;
  }
  const int rc = syncAndStatus(c);
  collectTimes(c);
  c->hostIter += steps;
  c->orderValid = false;
  return rc;
}

}  // extern "C"

namespace {
// Compaction of the objects flagged keep[j] = 1 in scratchA (current order;
// scratchC holds the same flags in slot order): survivors keep their
// relative slot order and are renumbered 0..n'-1.  The slot-indexed arrays
// are compacted through the roll-back buffer's positions and velocities,
// which hold nothing between calls.
int compactKept(ladds_gpu_ctx *c) {
  const int n = (int)c->n;
  uint32_t *keep = c->scratchA, *pos = c->scratchB, *aliveBySlot = c->scratchC, *newSlot = c->keys1;
  // exclusive scans: positions in the current order, new slot numbers in slot order
  enqueueExclusiveScan(c, keep, (size_t)n, pos);
  enqueueExclusiveScan(c, aliveBySlot, (size_t)n, newSlot);
  CK(cudaGetLastError());
  double *tRadius = c->snap.x;
  auto *tId = reinterpret_cast<uint64_t *>(c->snap.y), *tParent = reinterpret_cast<uint64_t *>(c->snap.z);
  k_compact<<<blocksFor(n, 256), 256, 0, c->st>>>(c->cur, c->alt, keep, pos, newSlot, n, tRadius, tId, tParent);
  uint32_t kept = 0, lastKeep = 0;
  CK(cudaMemcpyAsync(&kept, pos + (n - 1), sizeof(uint32_t), cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(&lastKeep, keep + (n - 1), sizeof(uint32_t), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  CK(cudaGetLastError());
  const size_t m = (size_t)kept + lastKeep;
  if (m) {  // back into the shared slot-indexed arrays
    CK(cudaMemcpyAsync(c->cur.radius, tRadius, m * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
    CK(cudaMemcpyAsync(c->cur.id, tId, m * sizeof(uint64_t), cudaMemcpyDeviceToDevice, c->st));
    CK(cudaMemcpyAsync(c->cur.parent, tParent, m * sizeof(uint64_t), cudaMemcpyDeviceToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
  }
  std::swap(c->cur, c->alt);
  c->n = m;
  c->orderValid = false;
  dropGraphs(c);
  return LADDS_OK;
}

// Conjunction scan of the current state (cell keys, sort, gather, pair scan),
// re-run with larger buffers after an overflow; sorted records in recs.
int scanState(ladds_gpu_ctx *c, const ScanConsts &sc, float cutF, std::vector<ladds_pair> &recs) {
  recs.clear();
  if (!c->n) return LADDS_OK;
  for (int attempt = 0; attempt < 5; ++attempt) {
    CK(cudaMemsetAsync(c->dCount, 0, sizeof(unsigned long long), c->st));
    CK(cudaMemsetAsync(c->dCandNeed, 0, sizeof(unsigned long long), c->st));
    CK(cudaMemsetAsync(c->rowCounts, 0, ((size_t)c->nRows + 1) * sizeof(uint32_t), c->st));
    k_cell_keys<<<blocksFor(c->n, 256), 256, 0, c->st>>>(c->cur.x, c->cur.y, c->cur.z, (int)c->n, c->grid,
                                                          c->keys0, c->rowCounts, c->scratchC);
    enqueueSort(c);
    enqueueCells(c);
    enqueueScanWith(c, c->st, sc, cutF, c->dIter, -1);  // records carry the index of the last integrated iteration
    int rc = syncAndStatus(c);
    collectTimes(c);
    if (rc) return rc;
    unsigned long long cnt = 0;
    bool overflow = false;
    rc = growIfOverflowed(c, &cnt, &overflow);
    if (rc) return rc;
    if (!overflow) {
      recs.resize(cnt);
      if (cnt) CK(cudaMemcpy(recs.data(), c->dPairs, cnt * sizeof(ladds_pair), cudaMemcpyDeviceToHost));
      c->orderValid = true;
      std::sort(recs.begin(), recs.end(), pairLess);
      return LADDS_OK;
    }
  }
  return fail(c, LADDS_ERR_CAPACITY, "scan buffers kept overflowing");
}
}  // namespace

extern "C" {

int ladds_gpu_scan(ladds_gpu_ctx *c, const ladds_scan_params *p, ladds_pair *out, size_t cap, size_t *nOut) {
  if (!c || !p || !nOut || !std::isfinite(p->dt) || !(p->cutoff > 0) || !(p->nearThresholdRel >= 0))
    return LADDS_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g_deviceMutex[c->dev & 63]);
  if (p->cutoff > c->cfg.cutoff)
    return fail(c, LADDS_ERR_INVALID_ARG, "scan cutoff larger than the cutoff the cell grid was built for");
  CK(cudaSetDevice(c->dev));
  ScanConsts sc;
  sc.cutoffSq = p->cutoff * p->cutoff;
  sc.dt = p->dt;
  sc.factor = p->collisionDistanceFactor / 1000.;
  sc.minDetectionRadius = p->minDetectionRadius;
  sc.evasionSq = p->evasionCutoff * p->evasionCutoff;
  sc.conjSq = p->conjunctionThreshold * p->conjunctionThreshold;
  sc.nearRel = p->nearThresholdRel;
  std::vector<ladds_pair> recs;
  const int rc = scanState(c, sc, prefilterRadius(p->cutoff, p->nearThresholdRel), recs);
  if (rc) return rc;
  *nOut = recs.size();
  if (recs.size() > cap || (!out && !recs.empty()))
    return fail(c, LADDS_ERR_CAPACITY, "output buffer too small for the conjunction records");
  if (!recs.empty()) std::memcpy(out, recs.data(), recs.size() * sizeof(ladds_pair));
  return LADDS_OK;
}

int ladds_gpu_conjunctions(ladds_gpu_ctx *c, double dtScan, ladds_pair *out, size_t cap, size_t *nOut,
                           size_t *nCollisions, size_t *nEvasions, size_t *nConjunctions) {
  if (!c || !nOut || !std::isfinite(dtScan)) return LADDS_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g_deviceMutex[c->dev & 63]);
  CK(cudaSetDevice(c->dev));
  std::vector<ladds_pair> recs;
  ScanConsts sc = c->sc;
  sc.dt = dtScan;
  const int rc = scanState(c, sc, c->cutF, recs);
  if (rc) return rc;
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
  // pair-buffer overflow and undone when the caller's buffer is too small.  A
  // one-iteration call changes only the positions and velocities of the
  // current buffer (its gather writes the other buffer), so they are all it
  // keeps; undoing it restores them and the buffer roles.
  const bool light = iterations == 1;
  const DevState curStart = c->cur, altStart = c->alt;
  if (light) {
    CK(copyDynamic(c->cur, c->snap, c->n, c->st));
  } else {
    CK(copyState(c->cur, c->snap, c->n, c->st));
  }
  const int64_t startIter = c->hostIter;
  auto rollBack = [&]() -> int {
    if (light) {
      c->cur = curStart;
      c->alt = altStart;
      CK(copyDynamic(c->snap, c->cur, c->n, c->st));
    } else {
      CK(copyState(c->snap, c->cur, c->n, c->st));
    }
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
    CK(cudaMemsetAsync(c->dCandNeed, 0, sizeof(unsigned long long), c->st));
    const bool graph = c->cfg.useGraphs && !c->profiling && iterations >= 1;
    const int64_t it0 = c->hostIter;
    if (graph) {
      // pass 1: capture the graphs this call needs (capture performs the host-side
      // buffer swaps; they are undone afterwards), so that no capture happens
      // between the timing events
      const DevState cur0 = c->cur, alt0 = c->alt;
      uint32_t *const sk0 = c->sortedKeys, *const pm0 = c->perm;
      const int par0 = c->sortParity;
      for (int done = 0; done < iterations;) {
        const int len = std::min(iterations - done, c->chunkSteps);
        const int bufs = (c->cur.x == c->homeX ? 0 : 1) | 2 * c->sortParity;
        const auto key = std::make_tuple(len, (int)((it0 + done) % k), bufs, c->n, c->pairCap);
        if (c->graphs.find(key) == c->graphs.end()) {
          CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
          enqueueChunk(c, it0 + done, len, k);
          cudaGraph_t gr = nullptr;
          CK(cudaStreamEndCapture(c->st, &gr));
          cudaGraphExec_t ex = nullptr;
          const cudaError_t ie = cudaGraphInstantiate(&ex, gr, 0);
          cudaGraphDestroy(gr);
          CK(ie);
          c->graphs.emplace(key, ex);
        } else {
          replaySwaps(c, it0 + done, len, k);
        }
        done += len;
      }
      c->cur = cur0;
      c->alt = alt0;
      if (c->sortParity != par0) swapSortSets(c);
      c->sortedKeys = sk0;
      c->perm = pm0;
      // pass 2: replay
      CK(cudaEventRecord(c->callStart, c->st));
      for (int done = 0; done < iterations;) {
        const int len = std::min(iterations - done, c->chunkSteps);
        const int bufs = (c->cur.x == c->homeX ? 0 : 1) | 2 * c->sortParity;
        const auto key = std::make_tuple(len, (int)((it0 + done) % k), bufs, c->n, c->pairCap);
        auto git = c->graphs.find(key);
        if (git == c->graphs.end()) return fail(c, LADDS_ERR_STATE, "graph cache inconsistent");
        replaySwaps(c, it0 + done, len, k);
        CK(cudaGraphLaunch(git->second, c->st));
        done += len;
      }
    } else {
      CK(cudaEventRecord(c->callStart, c->st));
      for (int done = 0; done < iterations;) {
        const int len = std::min(iterations - done, c->chunkSteps);
        enqueueChunk(c, it0 + done, len, k);
        done += len;
      }
    }
    CK(cudaEventRecord(c->callEnd, c->st));
    bool overflow = false;
    int rc = syncStatusAndGrow(c, &cnt, &overflow);
    collectTimes(c);
    if (rc) {
      const int rb = rollBack();
      return rb ? rb : rc;
    }
    if (!overflow) break;
    // a device record or candidate buffer overflowed: it has grown; roll back, run the batch again
    if (++retries > 4) {
      rollBack();
      return fail(c, LADDS_ERR_CAPACITY, "device scan buffers kept overflowing");
    }
    rc = rollBack();
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

}  // extern "C"


extern "C" {

int ladds_gpu_step_host(ladds_gpu_ctx *c, size_t n, const double *const in[6], double *const outState[6],
                        ladds_pair *out, size_t cap, size_t *nOut, ladds_step_stats *stats) {
  if (!c || !in || !outState || !nOut) return LADDS_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g_deviceMutex[c->dev & 63]);
  *nOut = 0;
  if (n != c->n) return fail(c, LADDS_ERR_INVALID_ARG, "step_host: n differs from the population size");
  for (int a = 0; a < 6; ++a)
    if (n && (!in[a] || !outState[a])) return fail(c, LADDS_ERR_INVALID_ARG, "null array pointer");
  CK(cudaSetDevice(c->dev));
  if (stats) std::memset(stats, 0, sizeof(*stats));
  c->pending.clear();
  const int k = c->cfg.timestepsPerCollisionDetection;
  const bool scan = (c->hostIter % k) == 0 && n;
  const int64_t startIter = c->hostIter;
  // the iteration's source buffer, in slot order: positions and velocities
  // from the host, the per-object constants and tags scattered out of the
  // current (cell-ordered) buffer
  const DevState S = c->snap;
  const int ni = (int)n;
  // any failure once work is enqueued: nothing of this call may still run when
  // it returns -- its copies into the caller's arrays and its kernels are
  // drained on all three streams -- and the iteration is not counted (the device
  // copy of the state is replaced by the next call's host state)
  auto abortCall = [&](int rc) {
    cudaStreamSynchronize(c->st2);
    cudaStreamSynchronize(c->st3);
    cudaStreamSynchronize(c->st);
    cudaMemcpyAsync(c->dIter, &startIter, sizeof(int64_t), cudaMemcpyHostToDevice, c->st);
    cudaStreamSynchronize(c->st);
    c->orderValid = false;
    return rc;
  };
#define CKS(call)                                                                                   \
  do {                                                                                              \
    cudaError_t e_ = (call);                                                                        \
    if (e_ != cudaSuccess)                                                                          \
      return abortCall(fail(c, LADDS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_))); \
  } while (0)
  CKS(cudaMemsetAsync(c->dCount, 0, 2 * sizeof(unsigned long long), c->st));
  CKS(cudaEventRecord(c->callStart, c->st));
  if (n) {
    const int g = blocksFor(n, 256);
    k_unpermute_f64<<<g, 256, 0, c->st>>>(c->cur.aom, c->cur.tag, ni, S.aom);
    k_unpermute_f64<<<g, 256, 0, c->st>>>(c->cur.bc, c->cur.tag, ni, S.bc);
    k_unpermute_tag<<<g, 256, 0, c->st>>>(c->cur.tag, ni, S.tag);
  }
  CKS(enqueueEphemeris(c, 1));
  if (scan) CKS(cudaMemsetAsync(c->rowCounts, 0, ((size_t)c->nRows + 1) * sizeof(uint32_t), c->st));
  // pageable arrays go through pinned staging, copied on all host threads
  // chunk by chunk (the CUDA driver's own staging of pageable copies is slower)
  bool stageIn[6] = {}, stageOut[6] = {}, anyIn = false, anyOut = false;
  for (int a = 0; a < 6 && n; ++a) {
    stageIn[a] = !isPinned(in[a]);
    stageOut[a] = !isPinned(outState[a]);
    anyIn |= stageIn[a];
    anyOut |= stageOut[a];
  }
  if ((anyIn || anyOut) && !ensurePinStage(c, n)) {  // no pinned memory to spare: the driver stages the copies
    for (int a = 0; a < 6; ++a) stageIn[a] = stageOut[a] = false;
    anyIn = anyOut = false;
  }
  double *pinIn[6], *pinOut[6];
  const double *src[6];
  double *dstHost[6];
  for (int a = 0; a < 6; ++a) {
    pinIn[a] = c->pinStage ? c->pinStage + (size_t)a * c->pinCap : nullptr;
    pinOut[a] = c->pinStage ? c->pinStage + (size_t)(6 + a) * c->pinCap : nullptr;
    src[a] = stageIn[a] ? pinIn[a] : in[a];
    dstHost[a] = stageOut[a] ? pinOut[a] : outState[a];
  }
  // chunks: host->device on st2, propagation on st, device->host on st3
  const int chunks = (int)std::max<size_t>(1, std::min<size_t>((size_t)kHostChunks, n / kHostChunkMin));
  // chunk starts on multiples of 256 objects keep every chunk's arrays 16-byte aligned (staged propagation)
  const size_t per = ((n + (size_t)chunks - 1) / (size_t)chunks + 255) / 256 * 256;
  double *const sArr[6] = {S.x, S.y, S.z, S.vx, S.vy, S.vz};
  int used = 0;
  for (int ch = 0; ch < chunks && n; ++ch) {
    const size_t lo = (size_t)ch * per;
    if (lo >= n) break;
    const size_t len = std::min(per, n - lo);
    if (anyIn) hostCopy(pinIn, in, stageIn, lo, len);
    for (int a = 0; a < 6; ++a)
      CKS(cudaMemcpyAsync(sArr[a] + lo, src[a] + lo, len * sizeof(double), cudaMemcpyHostToDevice, c->st2));
    CKS(cudaEventRecord(c->evPipe[ch], c->st2));
    CKS(cudaStreamWaitEvent(c->st, c->evPipe[ch], 0));
    DevState Sc = S;
    Sc.x += lo; Sc.y += lo; Sc.z += lo; Sc.vx += lo; Sc.vy += lo; Sc.vz += lo;
    Sc.aom += lo; Sc.bc += lo; Sc.tag += lo;
    launchPropagate(c, Sc, (int)len, 1, 0, scan, c->keys0 + lo, c->scratchC + lo);
    CKS(cudaEventRecord(c->evPipe[kHostChunks + ch], c->st));
    CKS(cudaStreamWaitEvent(c->st3, c->evPipe[kHostChunks + ch], 0));
    for (int a = 0; a < 6; ++a)
      CKS(cudaMemcpyAsync(dstHost[a] + lo, sArr[a] + lo, len * sizeof(double), cudaMemcpyDeviceToHost, c->st3));
    CKS(cudaEventRecord(c->evPipe[2 * kHostChunks + ch], c->st3));
    used = ch + 1;
  }
  k_advance<<<1, 32, 0, c->st>>>(c->dIter, 1);
  const DevState curStart = c->cur, altStart = c->alt;
  // the buffer roles when the call returns (on every path): S is the roll-back
  // buffer again and (cur, alt) the pair the captured graphs were made with;
  // the scan reads S as alt until then
  struct RoleGuard {
    ladds_gpu_ctx *c;
    DevState alt;
    bool on;
    ~RoleGuard() {
      if (on) c->alt = alt;
    }
  } roles{c, curStart, scan};
  ScanConsts sc = c->sc;
  sc.dt = c->cfg.deltaT * (double)k;
  if (scan) {
    // sort and gather from the slot-ordered buffer into the other buffer of the
    // pair, which becomes the current one (as after a scan of ladds_gpu_step)
    c->cur = S;
    c->alt = curStart;
    enqueueSort(c);
    c->alt = altStart;
    enqueueCells(c);  // gathers S into altStart, then cur = altStart, alt = S (the scan reads alt)
    enqueueScanWith(c, c->st, sc, c->cutF, c->dIterBase, 0);
  } else if (n) {
    // no scan: the new positions and velocities into the current buffer's order
    const int g = blocksFor(n, 256);
    double *const dst[6] = {c->cur.x, c->cur.y, c->cur.z, c->cur.vx, c->cur.vy, c->cur.vz};
    for (int a = 0; a < 6; ++a) k_permute_from_slots_f64<<<g, 256, 0, c->st>>>(sArr[a], c->cur.tag, ni, dst[a]);
  }
  if (used) {
    CKS(cudaEventRecord(c->evPipe[3 * kHostChunks], c->st3));
    CKS(cudaStreamWaitEvent(c->st, c->evPipe[3 * kHostChunks], 0));
  }
  CKS(cudaEventRecord(c->callEnd, c->st));
  // staged outputs: each chunk leaves the pinned buffer as soon as it is there
  for (int ch = 0; ch < used && anyOut; ++ch) {
    CKS(cudaEventSynchronize(c->evPipe[2 * kHostChunks + ch]));
    const size_t lo = (size_t)ch * per;
    hostCopy(outState, pinOut, stageOut, lo, std::min(per, n - lo));
  }
  unsigned long long cnt = 0;
  bool overflow = false;
  int rc = syncStatusAndGrow(c, &cnt, &overflow);
  collectTimes(c);
  if (rc) return abortCall(rc);
  int retries = 0;
  while (overflow) {  // the device buffers have grown: the scan alone runs again on the same state
    if (++retries > 4) return abortCall(fail(c, LADDS_ERR_STATE, "device scan buffers kept overflowing"));
    CKS(cudaMemsetAsync(c->dCount, 0, 2 * sizeof(unsigned long long), c->st));
    enqueueScanWith(c, c->st, sc, c->cutF, c->dIterBase, 0);
    rc = syncStatusAndGrow(c, &cnt, &overflow);
    collectTimes(c);
    if (rc) return abortCall(rc);
  }
  CKS(cudaStreamSynchronize(c->st3));
  float ms = 0;
  cudaEventElapsedTime(&ms, c->callStart, c->callEnd);
  std::vector<ladds_pair> recs(cnt);
  if (cnt) CKS(cudaMemcpy(recs.data(), c->dPairs, cnt * sizeof(ladds_pair), cudaMemcpyDeviceToHost));
  std::sort(recs.begin(), recs.end(), pairLess);
  c->hostIter += 1;
  if (scan) c->orderValid = true;
  if (stats) {
    stats->iterations = 1;
    stats->scans = scan ? 1 : 0;
    stats->records = cnt;
    stats->retries = (uint64_t)retries;
    stats->deviceMs = ms;
    for (const auto &p : recs) {
      stats->collisions += (p.flags & LADDS_PAIR_COLLISION) != 0;
      stats->evasions += (p.flags & LADDS_PAIR_EVASION) != 0;
      stats->conjunctions += (p.flags & LADDS_PAIR_CONJUNCTION) != 0;
    }
  }
  *nOut = recs.size();
  if (recs.size() > cap || (!out && !recs.empty())) {
    c->pending = std::move(recs);
    return fail(c, LADDS_ERR_CAPACITY, "output buffer too small: the records wait in ladds_gpu_pending_records");
  }
  if (!recs.empty()) std::memcpy(out, recs.data(), recs.size() * sizeof(ladds_pair));
  return LADDS_OK;
#undef CKS
}

int ladds_gpu_pending_records(ladds_gpu_ctx *c, ladds_pair *out, size_t cap, size_t *nOut) {
  if (!c || !nOut) return LADDS_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g_deviceMutex[c->dev & 63]);
  *nOut = c->pending.size();
  if (c->pending.size() > cap || (!out && !c->pending.empty()))
    return fail(c, LADDS_ERR_CAPACITY, "output buffer too small for the pending records");
  if (!c->pending.empty()) std::memcpy(out, c->pending.data(), c->pending.size() * sizeof(ladds_pair));
  c->pending.clear();
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

}  // extern "C"

namespace {
// ids of the objects flagged keep[j] == 0 in scratchA, in slot order (at most
// cap of them), gathered on the device: only the removed ones cross to the host
int removedIdsInSlotOrder(ladds_gpu_ctx *c, uint64_t *removedIds, size_t cap) {
  const int n = (int)c->n;
  unsigned *dCnt = reinterpret_cast<unsigned *>(c->dCandNeed) + 1;  // word 0 holds the removal count
  CK(cudaMemsetAsync(dCnt, 0, sizeof(unsigned), c->st));
  // keys0 / vals0 / scratchB are free between calls (scratchB is compactKept's output, written later)
  k_removed_ids<<<blocksFor(n, 256), 256, 0, c->st>>>(c->scratchA, c->cur.tag, c->cur.id, n, c->keys0, c->vals0,
                                                       c->scratchB, dCnt);
  CK(cudaGetLastError());
  unsigned m = 0;
  CK(cudaMemcpyAsync(&m, dCnt, sizeof(unsigned), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  std::vector<uint32_t> sl(m), lo(m), hi(m);
  if (m) {
    CK(cudaMemcpyAsync(sl.data(), c->keys0, m * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(lo.data(), c->vals0, m * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(hi.data(), c->scratchB, m * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
  }
  std::vector<uint32_t> order(m);
  for (uint32_t i = 0; i < m; ++i) order[i] = i;
  std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return sl[a] < sl[b]; });
  for (size_t w = 0; w < m && w < cap; ++w) removedIds[w] = ((uint64_t)hi[order[w]] << 32) | lo[order[w]];
  return LADDS_OK;
}

}  // namespace

extern "C" {

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
  unsigned *dBurnt = reinterpret_cast<unsigned *>(c->dCandNeed);  // scratch word (reset by every scan)
  CK(cudaMemsetAsync(dBurnt, 0, sizeof(unsigned), c->st));
  k_burnup_flags<<<blocksFor(n, 256), 256, 0, c->st>>>(c->cur.x, c->cur.y, c->cur.z, c->cur.tag, n, critSq,
                                                        c->scratchA, c->scratchC, dBurnt);
  unsigned burnt = 0;
  CK(cudaMemcpyAsync(&burnt, dBurnt, sizeof(unsigned), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  CK(cudaGetLastError());
  if (!burnt) return LADDS_OK;  // nothing burns up: the state, its order and the captured graphs stay
  if (removedIds) {  // ids of the removed objects, in slot order, before the compaction renumbers them
    const int rid = removedIdsInSlotOrder(c, removedIds, cap);
    if (rid) return rid;
  }
  int rc = compactKept(c);
  if (rc) return rc;
  if (nRemoved) *nRemoved = (size_t)n - c->n;
  return LADDS_OK;
}

int ladds_gpu_remove_escaping(ladds_gpu_ctx *c, size_t *nRemoved, uint64_t *removedIds, size_t cap) {
  if (!c) return LADDS_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g_deviceMutex[c->dev & 63]);
  if (nRemoved) *nRemoved = 0;
  if (!c->n) return LADDS_OK;
  CK(cudaSetDevice(c->dev));
  const int n = (int)c->n;
  const double3 lo = make_double3(c->cfg.boxMin[0], c->cfg.boxMin[1], c->cfg.boxMin[2]);
  const double3 hi = make_double3(c->cfg.boxMax[0], c->cfg.boxMax[1], c->cfg.boxMax[2]);
  unsigned *dOut = reinterpret_cast<unsigned *>(c->dCandNeed);  // scratch word (reset by every scan)
  CK(cudaMemsetAsync(dOut, 0, sizeof(unsigned), c->st));
  k_escape_flags<<<blocksFor(n, 256), 256, 0, c->st>>>(c->cur, n, lo, hi, c->scratchA, c->scratchC, dOut);
  unsigned escaped = 0;
  CK(cudaMemcpyAsync(&escaped, dOut, sizeof(unsigned), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  CK(cudaGetLastError());
  if (!escaped) return LADDS_OK;  // nobody leaves: the state, its order and the captured graphs stay
  if (removedIds) {  // ids of the removed objects, in slot order, before the compaction renumbers them
    const int rid = removedIdsInSlotOrder(c, removedIds, cap);
    if (rid) return rid;
  }
  int rc = compactKept(c);
  if (rc) return rc;
  if (nRemoved) *nRemoved = (size_t)n - c->n;
  return LADDS_OK;
}

int ladds_gpu_pack_layers(ladds_gpu_ctx *c, int32_t izLo, int32_t izHi, int remove, ladds_state_record *out,
                          size_t cap, size_t *nOut) {
  if (!c || !nOut || (cap && !out) || (!out && !remove))
    return fail(c, LADDS_ERR_INVALID_ARG, "pack_layers: bad argument");
  std::lock_guard<std::mutex> lk(g_deviceMutex[c->dev & 63]);
  *nOut = 0;
  if (!c->n || izHi <= izLo) return LADDS_OK;
  CK(cudaSetDevice(c->dev));
  if (cap) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, out) != cudaSuccess ||
        !((at.type == cudaMemoryTypeDevice && at.device == c->dev) || at.type == cudaMemoryTypeManaged)) {
      cudaGetLastError();
      return fail(c, LADDS_ERR_INVALID_ARG, "pack_layers: out must be device memory of the context's device");
    }
  }
  const int n = (int)c->n;
  // keys0 / vals0 are the sort's unsorted-key and source scratch (free between
  // calls); scratchA / scratchC take the removal flags of compactKept
  uint32_t *sel = c->keys0, *pos = c->vals0;
  auto *idx = reinterpret_cast<int32_t *>(c->scratchB);
  k_layer_flags<<<blocksFor(n, 256), 256, 0, c->st>>>(c->cur.z, c->cur.tag, n, c->grid, izLo, izHi, sel,
                                                       c->scratchA, c->scratchC);
  enqueueExclusiveScan(c, sel, (size_t)n, pos);
  CK(cudaGetLastError());
  uint32_t last[2] = {0, 0};
  CK(cudaMemcpyAsync(&last[0], pos + (n - 1), sizeof(uint32_t), cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(&last[1], sel + (n - 1), sizeof(uint32_t), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  const size_t count = (size_t)last[0] + last[1];
  *nOut = count;
  if (!count) return LADDS_OK;
  if (remove && !out) return compactKept(c);  // removed without being packed
  if (count > cap) return fail(c, LADDS_ERR_CAPACITY, "pack_layers: more particles than the output holds");
  k_selected_positions<<<blocksFor(n, 256), 256, 0, c->st>>>(sel, pos, n, idx);
  k_gather_records<<<blocksFor(count, 128), 128, 0, c->st>>>(c->cur, idx, (int)count, out);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->st));
  return remove ? compactKept(c) : LADDS_OK;
}

int ladds_gpu_append_records(ladds_gpu_ctx *c, const ladds_state_record *records, size_t m) {
  if (!c || (m && !records)) return fail(c, LADDS_ERR_INVALID_ARG, "append_records: bad argument");
  std::lock_guard<std::mutex> lk(g_deviceMutex[c->dev & 63]);
  if (!m) return LADDS_OK;
  CK(cudaSetDevice(c->dev));
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, records) != cudaSuccess ||
      !((at.type == cudaMemoryTypeDevice && at.device == c->dev) || at.type == cudaMemoryTypeManaged)) {
    cudaGetLastError();
    return fail(c, LADDS_ERR_INVALID_ARG, "append_records: records must be device memory of the context's device");
  }
  if (c->n + m > (size_t)kTagSlotMask) return fail(c, LADDS_ERR_TOO_LARGE, "append_records: too many particles");
  int rc = ensureCapacity(c, c->n + m);
  if (rc) return rc;
  // scratch words (reset by every scan): [0] bad records, [1] records with a parent
  unsigned *dBad = reinterpret_cast<unsigned *>(c->dCandNeed);
  CK(cudaMemsetAsync(dBad, 0, 2 * sizeof(unsigned), c->st));
  k_append_records<<<blocksFor(m, 128), 128, 0, c->st>>>(records, (int)m, c->cur, (uint32_t)c->n, dBad);
  CK(cudaGetLastError());
  unsigned flags[2] = {0, 0};
  CK(cudaMemcpyAsync(flags, dBad, 2 * sizeof(unsigned), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (flags[0]) return fail(c, LADDS_ERR_INVALID_ARG, "append_records: a record holds NaN/Inf or a bad activity state");
  if (flags[1]) c->anyParent = true;
  c->n += m;
  c->orderValid = false;
  dropGraphs(c);
  return LADDS_OK;
}

int ladds_gpu_truncate(ladds_gpu_ctx *c, size_t n0) {
  if (!c) return LADDS_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g_deviceMutex[c->dev & 63]);
  if (n0 >= c->n) return LADDS_OK;
  CK(cudaSetDevice(c->dev));
  k_truncate_flags<<<blocksFor(c->n, 256), 256, 0, c->st>>>(c->cur.tag, (int)c->n, (uint32_t)n0, c->scratchA,
                                                             c->scratchC);
  CK(cudaGetLastError());
  return compactKept(c);
}

int ladds_gpu_remove_slots(ladds_gpu_ctx *c, const uint32_t *slots, size_t m) {
  if (!c || (m && !slots)) return LADDS_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g_deviceMutex[c->dev & 63]);
  if (!m || !c->n) return LADDS_OK;
  for (size_t i = 0; i < m; ++i)
    if (slots[i] >= c->n) return fail(c, LADDS_ERR_INVALID_ARG, "slot out of range");
  CK(cudaSetDevice(c->dev));
  std::vector<uint8_t> mark(c->n, 0);
  for (size_t i = 0; i < m; ++i) mark[slots[i]] = 1;
  uint8_t *dMark = reinterpret_cast<uint8_t *>(c->scratchB);  // read before compactKept writes scratchB
  CK(cudaMemcpyAsync(dMark, mark.data(), c->n, cudaMemcpyHostToDevice, c->st));
  k_slot_mark_flags<<<blocksFor(c->n, 256), 256, 0, c->st>>>(c->cur.tag, (int)c->n, dMark, c->scratchA,
                                                              c->scratchC);
  return compactKept(c);
}

int ladds_gpu_select_layers(ladds_gpu_ctx *c, int32_t izLo, int32_t izHi, uint32_t *slots, size_t cap, size_t *n) {
  if (!c || !n || (cap && !slots)) return LADDS_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g_deviceMutex[c->dev & 63]);
  *n = 0;
  if (!c->n || izHi <= izLo) return LADDS_OK;
  CK(cudaSetDevice(c->dev));
  unsigned *dCount = reinterpret_cast<unsigned *>(c->dCandNeed);  // scratch word (reset by every scan)
  CK(cudaMemsetAsync(dCount, 0, sizeof(unsigned), c->st));
  k_select_layers<<<blocksFor(c->n, 256), 256, 0, c->st>>>(c->cur.z, c->cur.tag, (int)c->n, c->grid, izLo, izHi,
                                                            c->scratchA, dCount, (unsigned)c->n);
  unsigned cnt = 0;
  CK(cudaMemcpyAsync(&cnt, dCount, sizeof(unsigned), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  CK(cudaGetLastError());
  *n = cnt;
  if (cnt > cap) return fail(c, LADDS_ERR_CAPACITY, "select_layers: buffer too small");
  std::vector<uint32_t> h(cnt);
  if (cnt) CK(cudaMemcpy(h.data(), c->scratchA, cnt * sizeof(uint32_t), cudaMemcpyDeviceToHost));
  std::sort(h.begin(), h.end());
  std::copy(h.begin(), h.end(), slots);
  return LADDS_OK;
}

int ladds_gpu_layer_histogram(ladds_gpu_ctx *c, uint64_t *counts, size_t nLayers) {
  if (!c || !counts) return LADDS_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g_deviceMutex[c->dev & 63]);
  const size_t nz = (size_t)c->grid.n[2];
  if (nLayers < nz) return fail(c, LADDS_ERR_CAPACITY, "layer_histogram: fewer entries than cell layers");
  std::fill(counts, counts + nLayers, 0ull);
  if (!c->n) return LADDS_OK;
  CK(cudaSetDevice(c->dev));
  if (nz > c->cap) return fail(c, LADDS_ERR_CAPACITY, "layer_histogram: more cell layers than capacity");
  auto *dCounts = reinterpret_cast<unsigned long long *>(c->sortRec);  // cap entries of 8 B
  CK(cudaMemsetAsync(dCounts, 0, nz * sizeof(unsigned long long), c->st));
  k_layer_histogram<<<blocksFor(c->n, 256), 256, 0, c->st>>>(c->cur.z, c->cur.tag, (int)c->n, c->grid, dCounts);
  CK(cudaMemcpyAsync(counts, dCounts, nz * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  CK(cudaGetLastError());
  return LADDS_OK;
}

int ladds_gpu_set_halo(ladds_gpu_ctx *c, size_t haloStart) {
  if (!c) return LADDS_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g_deviceMutex[c->dev & 63]);
  const uint32_t h = haloStart >= (size_t)0xffffffffu ? 0xffffffffu : (uint32_t)haloStart;
  if (h != c->haloStart) dropGraphs(c);  // captured scans carry the old value
  c->haloStart = h;
  return LADDS_OK;
}

int ladds_gpu_functor_pairs(ladds_gpu_ctx *c, const ladds_scan_params *p, size_t nPairs, const ladds_object *first,
                            const ladds_object *second, ladds_pair *out, size_t cap, size_t *nOut) {
  if (!c || !p || !nOut || (nPairs && (!first || !second)) || nPairs > (size_t)INT32_MAX)
    return LADDS_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(g_deviceMutex[c->dev & 63]);
  *nOut = 0;
  if (!nPairs) return LADDS_OK;
  for (size_t k = 0; k < nPairs; ++k)
    for (const ladds_object *o : {&first[k], &second[k]})
      if (o->activity < 0 || o->activity > 2 || o->slot > kTagSlotMask)
        return fail(c, LADDS_ERR_INVALID_ARG, "object activity or slot out of range");
  CK(cudaSetDevice(c->dev));
  if (nPairs > c->objCap) {
    if (c->dObj) cudaFree(c->dObj);
    c->dObj = nullptr;
    c->objCap = 0;
    if (cudaMalloc(&c->dObj, 2 * nPairs * sizeof(ladds_object)) != cudaSuccess) {
      cudaGetLastError();
      return fail(c, LADDS_ERR_ALLOC, "device allocation failed (pair objects)");
    }
    c->objCap = nPairs;
  }
  CK(cudaMemcpyAsync(c->dObj, first, nPairs * sizeof(ladds_object), cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->dObj + nPairs, second, nPairs * sizeof(ladds_object), cudaMemcpyHostToDevice, c->st));
  ScanConsts sc;
  sc.cutoffSq = p->cutoff * p->cutoff;
  sc.dt = p->dt;
  sc.factor = p->collisionDistanceFactor / 1000.;
  sc.minDetectionRadius = p->minDetectionRadius;
  sc.evasionSq = p->evasionCutoff * p->evasionCutoff;
  sc.conjSq = p->conjunctionThreshold * p->conjunctionThreshold;
  sc.nearRel = p->nearThresholdRel;
  std::vector<ladds_pair> recs;
  for (int attempt = 0; attempt < 3; ++attempt) {
    CK(cudaMemsetAsync(c->dCount, 0, sizeof(unsigned long long), c->st));
    k_functor_pairs<<<blocksFor(nPairs, 256), 256, 0, c->st>>>(c->dObj, c->dObj + nPairs, (int)nPairs, sc,
                                                                c->dPairs, c->dCount,
                                                                (unsigned long long)c->pairCap);
    CK(cudaStreamSynchronize(c->st));
    CK(cudaGetLastError());
    unsigned long long cnt = 0;
    CK(cudaMemcpy(&cnt, c->dCount, sizeof(cnt), cudaMemcpyDeviceToHost));
    if (cnt <= c->pairCap) {
      recs.resize(cnt);
      if (cnt) CK(cudaMemcpy(recs.data(), c->dPairs, cnt * sizeof(ladds_pair), cudaMemcpyDeviceToHost));
      break;
    }
    const int rc = ensurePairCapacity(c, (size_t)cnt);
    if (rc) return rc;
  }
  std::sort(recs.begin(), recs.end(), pairLess);
  *nOut = recs.size();
  if (recs.size() > cap || (!out && !recs.empty()))
    return fail(c, LADDS_ERR_CAPACITY, "output buffer too small for the pair records");
  if (!recs.empty()) std::memcpy(out, recs.data(), recs.size() * sizeof(ladds_pair));
  return LADDS_OK;
}

}  // extern "C"

// ----------------------------------------------------------------------------
// Autotuner: cell size, block shapes and the captured chunk length.
namespace {

// one timed trial of `cfg` (+ chunk length) on a copy of c's population
int tuneTrial(ladds_gpu_ctx *c, const ladds_gpu_config &cfg, int chunk, int steps, ladds_tune_trial &t) {
  ladds_gpu_ctx *tc = nullptr;
  int rc = ladds_gpu_create(&cfg, &tc);
  if (rc) return fail(c, rc, "autotune: a trial context could not be created");
  tc->chunkSteps = chunk;
  rc = ensureCapacity(tc, c->n);
  if (!rc && c->n) {
    const cudaError_t e = copyState(c->cur, tc->cur, c->n, c->st);
    if (e != cudaSuccess) rc = fail(c, LADDS_ERR_CUDA, cudaGetErrorString(e));
  }
  if (!rc && cudaStreamSynchronize(c->st) != cudaSuccess) rc = fail(c, LADDS_ERR_CUDA, "autotune: state copy");
  if (!rc) {
    tc->n = c->n;
    rc = ladds_gpu_set_iteration(tc, c->hostIter);
  }
  std::vector<ladds_pair> recs((size_t)1 << 16);
  ladds_step_stats st{};
  for (int pass = 0; pass < 2 && !rc; ++pass) {  // warm-up (captures the graphs), then the timed run
    const int n = pass == 0 ? std::min(steps, 2 * chunk) : steps;
    size_t got = 0;
    rc = ladds_gpu_step(tc, n, recs.data(), recs.size(), &got, &st);
    if (rc == LADDS_ERR_CAPACITY) {
      recs.resize(got);
      rc = ladds_gpu_step(tc, n, recs.data(), recs.size(), &got, &st);
    }
    if (rc) rc = fail(c, rc, std::string("autotune trial: ") + ladds_gpu_last_error(tc));
  }
  if (!rc) {
    t.cellSize = tc->grid.cellSize;
    t.reach = tc->grid.reach;
    t.propagateBlock = cfg.propagateBlock;
    t.scanBlock = cfg.scanBlock;
    t.chunkSteps = chunk;
    t.scanScreen = cfg.scanScreen;
    t.walkForm = cfg.walkForm;
    t.msPerStep = st.deviceMs / std::max(steps, 1);
  }
  ladds_gpu_destroy(tc);
  return rc;
}

}  // namespace

extern "C" {

int ladds_gpu_autotune(ladds_gpu_ctx *c, int stepsPerTrial, ladds_tune_trial *trials, size_t cap, size_t *nTrials,
                       ladds_tune_trial *best) {
  if (!c || stepsPerTrial < 1 || !best || (cap && !trials)) return fail(c, LADDS_ERR_INVALID_ARG, "autotune: bad argument");
  std::vector<ladds_tune_trial> all;
  ladds_gpu_config cfg = c->cfg;
  cfg.pairCapacity = c->pairCap;
  cfg.useGraphs = 1;
  ladds_tune_trial bestT{};
  bestT.msPerStep = INFINITY;
  int bestChunk = c->chunkSteps;
  auto run = [&](const ladds_gpu_config &k, int chunk) -> int {
    ladds_tune_trial t{};
    const int rc = tuneTrial(c, k, chunk, stepsPerTrial, t);
    if (rc) return rc;
    all.push_back(t);
    if (t.msPerStep < bestT.msPerStep) {
      bestT = t;
      cfg = k;
      bestChunk = chunk;
    }
    return LADDS_OK;
  };
  // 0. where full candidate buffers are screened (the population's density
  //    decides), at the current cell edge
  {
    const ladds_gpu_config base = cfg;
    for (int screen : {LADDS_SCREEN_LISTS, LADDS_SCREEN_BUFFER})
      for (int walk : {LADDS_WALK_GROUPED, LADDS_WALK_ROWS}) {
        ladds_gpu_config k = base;
        k.scanScreen = screen;
        k.walkForm = walk;
        const int rc = run(k, bestChunk);
        if (rc) return rc;
      }
  }
  // 1. cell edge in [20, 160] km: cutoff / R (neighbour reach R = 1..4) and
  //    coarser cells 1.5 and 2 cutoffs wide (reach 1); the current edge is
  //    measured already
  {
    const ladds_gpu_config base = cfg;
    std::vector<double> cells = {base.cellSize};
    for (int R = 1; R <= 4; ++R) cells.push_back(base.cutoff * (1.0 + 1e-6) / R);
    cells.push_back(1.5 * base.cutoff);
    cells.push_back(2.0 * base.cutoff);
    for (size_t i = 1; i < cells.size(); ++i) {
      const double cs = cells[i];
      if (cs < 20.0 || cs > 160.0) continue;
      if (i == 1 && base.cellSize <= 0) continue;  // the default edge: measured as the current one
      if (i > 1 && cs == base.cellSize) continue;
      ladds_gpu_config k = base;
      k.cellSize = cs;
      const int rc = run(k, bestChunk);
      if (rc) return rc;
    }
  }
  // 1b. the other walk form at the chosen cell edge (the form that suits a
  //     cell edge depends on the items per window, which the edge sets)
  {
    const ladds_gpu_config base = cfg;
    ladds_gpu_config k = base;
    k.walkForm = base.walkForm == LADDS_WALK_ROWS ? LADDS_WALK_GROUPED : LADDS_WALK_ROWS;
    const int rc = run(k, bestChunk);
    if (rc) return rc;
  }
  // 2. block shapes of the propagation and of the pair evaluation
  {
    const ladds_gpu_config base = cfg;
    for (int pb : {128, 256})
      for (int sb : {128, 256}) {
        ladds_gpu_config k = base;
        k.propagateBlock = pb;
        k.scanBlock = sb;
        if ((pb == base.propagateBlock || (pb == 256 && base.propagateBlock == 0)) &&
            (sb == base.scanBlock || (sb == 256 && base.scanBlock == 0)))
          continue;  // measured already
        const int rc = run(k, bestChunk);
        if (rc) return rc;
      }
  }
  // 3. iterations per captured chunk
  {
    const ladds_gpu_config base = cfg;
    for (int chunk : {32, 64, 128}) {
      if (chunk == bestChunk) continue;
      const int rc = run(base, chunk);
      if (rc) return rc;
    }
  }
  // apply the best configuration to the context (its state is untouched)
  std::lock_guard<std::mutex> lk(g_deviceMutex[c->dev & 63]);
  CK(cudaSetDevice(c->dev));
  CK(cudaStreamSynchronize(c->st));
  const bool regrid = cfg.cellSize != c->cfg.cellSize;
  c->cfg.cellSize = cfg.cellSize;
  c->cfg.propagateBlock = cfg.propagateBlock;
  c->cfg.scanBlock = cfg.scanBlock;
  c->cfg.scanScreen = cfg.scanScreen;
  c->cfg.walkForm = cfg.walkForm;
  c->chunkSteps = bestChunk;
  dropGraphs(c);
  if (regrid) {
    freeGridBuffers(c);
    int rc = buildGrid(c);
    if (!rc) rc = allocGridBuffers(c);
    if (rc) return rc;
    if (c->cap) {  // the row-start scan's partial sums are sized by max(objects, rows)
      const size_t scanLen = std::max(c->cap + 1, (size_t)c->nRows + 1);
      const size_t wsWords = 4 * (scanLen / kScanBlock + 2) + 4 * kScanBlock;
      if (c->scanWs) cudaFree(c->scanWs);
      c->scanWs = nullptr;
      if (cudaMalloc(&c->scanWs, wsWords * sizeof(uint32_t)) != cudaSuccess) {
        cudaGetLastError();
        return fail(c, LADDS_ERR_ALLOC, "autotune: scan workspace");
      }
    }
    c->orderValid = false;
  }
  *best = bestT;
  if (nTrials) *nTrials = all.size();
  for (size_t i = 0; i < all.size() && i < cap; ++i) trials[i] = all[i];
  return LADDS_OK;
}

}  // extern "C"

// ----------------------------------------------------------------------------
// Adjoint of the propagation for conjunction pairs (kernels in adjoint.cuh).
namespace {

template <typename T>
int ensureDev(ladds_gpu_ctx *c, T *&p, size_t &cap, size_t need) {
  if (need <= cap && p) return LADDS_OK;
  if (p) cudaFree(p);
  p = nullptr;
  cap = 0;
  if (cudaMalloc(&p, need * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    p = nullptr;
    return fail(c, LADDS_ERR_ALLOC, "device allocation for the adjoint pair batch failed");
  }
  cap = need;
  return LADDS_OK;
}

// buffers of nPairs pairs, `steps` steps, checkpoints every ck; ephemeris of the steps
int adjPrepare(ladds_gpu_ctx *c, size_t nPairs, int steps, int ck, bool backward) {
  auto &A = c->adj;
  const size_t nObj = 2 * nPairs;
  size_t objCap = A.objCap;
  int rc;
  if (nObj > A.objCap) {
    size_t cap0 = 0, cap1 = 0, cap2 = 0, cap3 = 0, cap4 = 0, cap5 = 0, cap6 = 0;
    if ((rc = ensureDev(c, A.st, cap0, 6 * nObj)) || (rc = ensureDev(c, A.bc, cap1, nObj)) ||
        (rc = ensureDev(c, A.aom, cap2, nObj)) || (rc = ensureDev(c, A.miss, cap3, nPairs)) ||
        (rc = ensureDev(c, A.grad, cap4, 7 * nObj)) || (rc = ensureDev(c, A.arg, cap5, nPairs)) ||
        (rc = ensureDev(c, A.off, cap6, 6 * nPairs))) {
      A.objCap = 0;
      return rc;
    }
    objCap = nObj;
  }
  A.objCap = objCap;
  const size_t nSeg = (size_t)((steps + ck - 1) / ck);
  if ((rc = ensureDev(c, A.ckpt, A.ckptCap, nSeg * 6 * nObj))) return rc;
  if (backward && (rc = ensureDev(c, A.rec, A.recCap, (size_t)ck * 15 * nObj))) return rc;
  if ((rc = ensureDev(c, A.eph, A.ephCap, (size_t)3 * steps))) return rc;
  return LADDS_OK;
}

int adjEphemeris(ladds_gpu_ctx *c, int steps) {
  k_ephemeris<<<blocksFor((size_t)3 * steps, 128), 128, 0, c->st>>>(c->adj.eph, steps, 0, c->cfg.startTime,
                                                                     c->cfg.deltaT, c->pc.hc1, c->pc.hc2,
                                                                     c->cfg.epochJD, c->theta0);
  CK(cudaGetLastError());
  return LADDS_OK;
}

}  // namespace

extern "C" {

int ladds_gpu_adjoint_forward(ladds_gpu_ctx *c, const ladds_adjoint_pair *pairs, size_t nPairs, int steps,
                              int checkpointEvery, double *missSq, int32_t *tcaStep, double *loss,
                              double *deviceMs) {
  if (!c || (nPairs && !pairs) || steps < 1 || checkpointEvery < 1 || nPairs > (size_t)(1 << 29))
    return fail(c, LADDS_ERR_INVALID_ARG, "adjoint_forward: bad argument");
  std::lock_guard<std::mutex> lk(g_deviceMutex[c->dev & 63]);
  CK(cudaSetDevice(c->dev));
  auto &A = c->adj;
  A.forwardDone = false;
  int rc = adjPrepare(c, nPairs, steps, checkpointEvery, false);
  if (rc) return rc;
  const size_t nObj = 2 * nPairs;
  // pairs (AoS) -> object SoA
  std::vector<double> st(6 * nObj), bc(nObj), aom(nObj);
  for (size_t p = 0; p < nPairs; ++p) {
    const ladds_adjoint_pair &q = pairs[p];
    for (int k = 0; k < 3; ++k) {
      st[k * nObj + 2 * p] = q.rA[k];
      st[(3 + k) * nObj + 2 * p] = q.vA[k];
      st[k * nObj + 2 * p + 1] = q.rB[k];
      st[(3 + k) * nObj + 2 * p + 1] = q.vB[k];
    }
    bc[2 * p] = q.bcInvA;
    bc[2 * p + 1] = q.bcInvB;
    aom[2 * p] = q.aomA;
    aom[2 * p + 1] = q.aomB;
  }
  if (nObj) {
    CK(cudaMemcpyAsync(A.st, st.data(), st.size() * sizeof(double), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(A.bc, bc.data(), bc.size() * sizeof(double), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(A.aom, aom.data(), aom.size() * sizeof(double), cudaMemcpyHostToDevice, c->st));
  }
  if ((rc = adjEphemeris(c, steps))) return rc;
  CK(cudaEventRecord(c->callStart, c->st));
  if (nObj)
    k_adj_forward<<<blocksFor(nObj, kAdjObjs), kAdjWarps * 32, 0, c->st>>>(A.st, A.bc, A.aom, (int)nObj, steps, checkpointEvery,
                                                           A.eph, c->pc, c->cfg.deltaT, A.ckpt, A.miss, A.arg);
  CK(cudaEventRecord(c->callEnd, c->st));
  CK(cudaGetLastError());
  std::vector<double> miss(nPairs);
  std::vector<int> arg(nPairs);
  if (nPairs) {
    CK(cudaMemcpyAsync(miss.data(), A.miss, nPairs * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(arg.data(), A.arg, nPairs * sizeof(int), cudaMemcpyDeviceToHost, c->st));
  }
  CK(cudaStreamSynchronize(c->st));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, c->callStart, c->callEnd));
  if (deviceMs) *deviceMs = ms;
  double sum = 0.0;
  for (size_t p = 0; p < nPairs; ++p) {
    if (missSq) missSq[p] = miss[p];
    if (tcaStep) tcaStep[p] = arg[p];
    if (arg[p] > 0) sum += miss[p];
  }
  if (loss) *loss = sum;
  A.nPairs = nPairs;
  A.steps = steps;
  A.ck = checkpointEvery;
  A.forwardDone = true;
  return LADDS_OK;
}

int ladds_gpu_adjoint_backward(ladds_gpu_ctx *c, double *dL_dx0, double *dL_dbc, double *deviceMs) {
  if (!c || !dL_dx0 || !dL_dbc) return fail(c, LADDS_ERR_INVALID_ARG, "adjoint_backward: null output");
  auto &A = c->adj;
  if (!A.forwardDone) return fail(c, LADDS_ERR_STATE, "adjoint_backward needs a preceding adjoint_forward");
  std::lock_guard<std::mutex> lk(g_deviceMutex[c->dev & 63]);
  CK(cudaSetDevice(c->dev));
  int rc = adjPrepare(c, A.nPairs, A.steps, A.ck, true);
  if (rc) return rc;
  const size_t nObj = 2 * A.nPairs;
  CK(cudaEventRecord(c->callStart, c->st));
  if (nObj)
    k_adj_backward<<<blocksFor(nObj, kAdjObjs), kAdjWarps * 32, 0, c->st>>>(A.bc, A.aom, (int)nObj, A.steps, A.ck, A.eph, c->pc,
                                                            c->cfg.deltaT, A.ckpt, A.arg, A.rec, A.grad);
  CK(cudaEventRecord(c->callEnd, c->st));
  CK(cudaGetLastError());
  std::vector<double> g(7 * nObj);
  if (nObj) CK(cudaMemcpyAsync(g.data(), A.grad, g.size() * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, c->callStart, c->callEnd));
  if (deviceMs) *deviceMs = ms;
  for (size_t p = 0; p < A.nPairs; ++p) {
    for (int k = 0; k < 6; ++k) {
      dL_dx0[12 * p + k] = g[k * nObj + 2 * p];
      dL_dx0[12 * p + 6 + k] = g[k * nObj + 2 * p + 1];
    }
    dL_dbc[2 * p] = g[6 * nObj + 2 * p];
    dL_dbc[2 * p + 1] = g[6 * nObj + 2 * p + 1];
  }
  return LADDS_OK;
}

int ladds_gpu_adjoint_make_pairs(ladds_gpu_ctx *c, uint64_t seed, size_t nPairs, int steps,
                                 ladds_adjoint_pair *out, int32_t *tcaStep) {
  if (!c || (nPairs && !out) || steps < 2 || nPairs > (size_t)(1 << 29))
    return fail(c, LADDS_ERR_INVALID_ARG, "adjoint_make_pairs: bad argument");
  std::lock_guard<std::mutex> lk(g_deviceMutex[c->dev & 63]);
  CK(cudaSetDevice(c->dev));
  auto &A = c->adj;
  A.forwardDone = false;
  int rc = adjPrepare(c, nPairs, steps, steps, false);
  if (rc) return rc;
  const size_t nObj = 2 * nPairs;
  std::vector<double> st(6 * nObj), bc(nObj), aom(nObj), off(6 * nPairs);
  std::vector<int> tca(nPairs);
  for (size_t p = 0; p < nPairs; ++p) {
    double sa[6], sb[6], dr[3], dv[3];
    adjointPairDraw(seed, p, c->cfg.deltaT, steps, sa, sb, bc[2 * p], aom[2 * p], bc[2 * p + 1], aom[2 * p + 1],
                    dr, dv, tca[p]);
    for (int k = 0; k < 6; ++k) {
      st[k * nObj + 2 * p] = sa[k];
      st[k * nObj + 2 * p + 1] = sb[k];
    }
    for (int k = 0; k < 3; ++k) {
      off[6 * p + k] = dr[k];
      off[6 * p + 3 + k] = dv[k];
    }
  }
  int *dTca = A.arg;  // the forward's argmin buffer serves as scratch here
  if (nObj) {
    CK(cudaMemcpyAsync(A.st, st.data(), st.size() * sizeof(double), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(A.bc, bc.data(), bc.size() * sizeof(double), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(A.aom, aom.data(), aom.size() * sizeof(double), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(A.off, off.data(), off.size() * sizeof(double), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(dTca, tca.data(), tca.size() * sizeof(int), cudaMemcpyHostToDevice, c->st));
  }
  if ((rc = adjEphemeris(c, steps))) return rc;
  PropConsts back = c->pc;
  back.hc1 = -back.hc1;
  back.hc2 = -back.hc2;
  back.hd1 = -back.hd1;
  back.hd2 = -back.hd2;
  if (nPairs)
    k_adj_make_pairs<<<blocksFor(nPairs, 128), 128, 0, c->st>>>(A.st, A.bc, A.aom, (int)nPairs, dTca, A.off, A.eph,
                                                                c->pc, back);
  CK(cudaGetLastError());
  if (nObj) CK(cudaMemcpyAsync(st.data(), A.st, st.size() * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  for (size_t p = 0; p < nPairs; ++p) {
    ladds_adjoint_pair &q = out[p];
    for (int k = 0; k < 3; ++k) {
      q.rA[k] = st[k * nObj + 2 * p];
      q.vA[k] = st[(3 + k) * nObj + 2 * p];
      q.rB[k] = st[k * nObj + 2 * p + 1];
      q.vB[k] = st[(3 + k) * nObj + 2 * p + 1];
    }
    q.bcInvA = bc[2 * p];
    q.bcInvB = bc[2 * p + 1];
    q.aomA = aom[2 * p];
    q.aomB = aom[2 * p + 1];
    if (tcaStep) tcaStep[p] = tca[p];
  }
  return LADDS_OK;
}

}  // extern "C"

// ----------------------------------------------------------------------------
// Cell sort without allocation (ladds_gpu_cell_sort_noalloc).
//
// For callers that cannot allocate device memory: processes in which another
// framework's caching allocator (JAX, PyTorch) has reserved nearly all of HBM,
// so that cudaMalloc fails, and callers on a per-iteration latency path that
// cannot take the implicit device synchronisation of cudaMalloc / cudaFree.
// All scratch of the sort (row counts and cursors, row-start table, sort
// records, source indices, long-row list, scan partial sums, status word)
// lives in one file-scope device array of fixed size; the caller supplies the
// keys and the output buffers.  Every call shares the array and it keeps the
// last call's contents, so each call clears what must start at zero, and calls
// that overlap on the GPU (other streams, other host threads) race.
namespace {

constexpr size_t naRound(size_t b) { return (b + 255) & ~(size_t)255; }
constexpr size_t kNaMaxObjects = LADDS_NOALLOC_SORT_MAX_OBJECTS;
constexpr size_t kNaMaxRows = LADDS_NOALLOC_SORT_MAX_ROWS;
constexpr size_t kNaScanBlocks = (kNaMaxRows + 1 + kScanBlock - 1) / kScanBlock;
static_assert(kNaScanBlocks <= (size_t)kScanBlock, "two scan levels must cover the row table");
// byte offsets inside the scratch array
constexpr size_t kNaRec = 0;                                                   // u64 per object
constexpr size_t kNaSrc = kNaRec + naRound(8 * kNaMaxObjects);                 // u32 per object
constexpr size_t kNaCounts = kNaSrc + naRound(4 * kNaMaxObjects);              // counts | cursors
constexpr size_t kNaRowStart = kNaCounts + naRound(8 * (kNaMaxRows + 1));      // u32 per row + 1
constexpr size_t kNaLong = kNaRowStart + naRound(4 * (kNaMaxRows + 1));        // long-row list
constexpr size_t kNaMisc = kNaLong + naRound(4 * kNaMaxRows);                  // longCount, status
constexpr size_t kNaScan = kNaMisc + 256;                                      // scan partial sums
constexpr size_t kNaBytes = kNaScan + naRound(4 * (2 * (kNaScanBlocks + 1) + 2));

static __device__ __align__(256) unsigned char g_noallocSortScratch[kNaBytes];

struct NaDevice {
  unsigned char *scratch = nullptr;  // device address of g_noallocSortScratch on this device
  int sms = 0;
};
NaDevice g_naDevice[64];
std::mutex g_naMutex;

void naMessage(char *msg, size_t cap, const char *text) {
  if (msg && cap) std::snprintf(msg, cap, "%s", text);
}

// status bits: 1 = a key beyond the grid, 2 = inconsistent row counts
__global__ void __launch_bounds__(kBucketThreads) k_na_count(const uint32_t *__restrict__ keys, int n, uint32_t nx,
                                                             uint32_t nRows, uint32_t *__restrict__ rowCount,
                                                             unsigned *__restrict__ status) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t row = 0xffffffffu;
  if (j < n) {
    row = keys[j] / nx;
    if (row >= nRows) {
      atomicOr(status, 1u);
      row = 0xffffffffu;
    }
  }
  const bool valid = row != 0xffffffffu;
  const uint32_t peers = __match_any_sync(0xffffffffu, row);
  if (valid && (__ffs(peers) - 1) == (int)(threadIdx.x & 31)) atomicAdd(&rowCount[row], (uint32_t)__popc(peers));
}

// sort record ix << 32 | j and source j of every object j (the index in keys)
__global__ void __launch_bounds__(kBucketThreads) k_na_scatter(const uint32_t *__restrict__ keys, int n, uint32_t nx,
                                                               uint32_t nRows, const uint32_t *__restrict__ rowStart,
                                                               uint32_t *__restrict__ rowCursor,
                                                               unsigned long long *__restrict__ rec,
                                                               uint32_t *__restrict__ src,
                                                               unsigned *__restrict__ status) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const uint32_t key = j < n ? keys[j] : 0u;
  uint32_t row = j < n ? key / nx : 0xffffffffu;
  if (row >= nRows) row = 0xffffffffu;  // counted as an error by k_na_count
  const bool valid = row != 0xffffffffu;
  const uint32_t peers = __match_any_sync(0xffffffffu, row);
  const int leader = __ffs(peers) - 1;
  uint32_t base = 0;
  if (valid && lane == leader) base = atomicAdd(&rowCursor[row], (uint32_t)__popc(peers));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (!valid) return;
  const uint32_t pos = rowStart[row] + base + (uint32_t)__popc(peers & laneMaskLt());
  if (pos >= rowStart[row + 1]) {
    atomicOr(status, 2u);
    return;
  }
  rec[pos] = ((unsigned long long)(key - row * nx) << 32) | (uint32_t)j;
  src[pos] = (uint32_t)j;
}

struct DeviceGuard {
  int prev = -1;
  cudaError_t status;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    status = cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

}  // namespace

extern "C" {

int ladds_gpu_cell_sort_noalloc(int device, void *stream, const uint32_t *keys, size_t n, const int32_t dims[3],
                                uint32_t *sortedKeys, uint32_t *order, uint32_t *rowStart, char *errMsg,
                                size_t errMsgCap) {
  naMessage(errMsg, errMsgCap, "");
  if (!dims || device < 0 || device >= 64 || (n && (!keys || !sortedKeys || !order))) {
    naMessage(errMsg, errMsgCap, "invalid argument: null pointer or device index");
    return LADDS_ERR_INVALID_ARG;
  }
  if (dims[0] < 1 || dims[1] < 1 || dims[2] < 1 ||
      (uint64_t)dims[0] * (uint64_t)dims[1] * (uint64_t)dims[2] > (1ull << 32)) {
    naMessage(errMsg, errMsgCap, "invalid argument: grid dimensions must be >= 1 with at most 2^32 cells");
    return LADDS_ERR_INVALID_ARG;
  }
  const uint64_t nRows64 = (uint64_t)dims[1] * (uint64_t)dims[2];
  if (n > kNaMaxObjects || nRows64 > kNaMaxRows) {
    char text[160];
    std::snprintf(text, sizeof(text),
                  "too large: %zu objects and %llu cell rows exceed the fixed scratch maximum of %zu objects / "
                  "%zu rows",
                  n, (unsigned long long)nRows64, kNaMaxObjects, kNaMaxRows);
    naMessage(errMsg, errMsgCap, text);
    return LADDS_ERR_TOO_LARGE;
  }
  // an error that earlier work left in this thread's CUDA state is not this
  // call's: report it without clearing it
  if (const cudaError_t pending = cudaPeekAtLastError(); pending != cudaSuccess) {
    char text[200];
    std::snprintf(text, sizeof(text), "a CUDA error of earlier work is pending (not cleared): %s",
                  cudaGetErrorString(pending));
    naMessage(errMsg, errMsgCap, text);
    return LADDS_ERR_CUDA;
  }
  DeviceGuard guard(device);
  if (guard.status != cudaSuccess) {
    cudaGetLastError();
    naMessage(errMsg, errMsgCap, cudaGetErrorString(guard.status));
    return guard.status == cudaErrorInvalidDevice || guard.status == cudaErrorNoDevice ? LADDS_ERR_NO_DEVICE
                                                                                        : LADDS_ERR_CUDA;
  }
  // the call waits for its stream and reads a status word back: it cannot be
  // part of a stream capture
  cudaStream_t s = (cudaStream_t)stream;
  cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
  if (const cudaError_t ce = cudaStreamIsCapturing(s, &capturing); ce != cudaSuccess) {
    cudaGetLastError();
    naMessage(errMsg, errMsgCap, cudaGetErrorString(ce));
    return LADDS_ERR_CUDA;
  }
  if (capturing != cudaStreamCaptureStatusNone) {
    naMessage(errMsg, errMsgCap, "invalid argument: the stream is capturing; this call synchronises its stream");
    return LADDS_ERR_INVALID_ARG;
  }
  NaDevice &d = g_naDevice[device];
  {
    std::lock_guard<std::mutex> lk(g_naMutex);
    if (!d.scratch) {  // set-up, once per device, with that device current
      int sms = 0;
      unsigned char *ptr = nullptr;
      const cudaError_t e1 = cudaGetSymbolAddress((void **)&ptr, g_noallocSortScratch);
      const cudaError_t e2 = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
      if (e1 != cudaSuccess || e2 != cudaSuccess || !ptr) {
        cudaGetLastError();
        naMessage(errMsg, errMsgCap, cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
        return LADDS_ERR_CUDA;
      }
      d.sms = std::max(sms, 1);
      d.scratch = ptr;
    }
  }
  const uint32_t nx = (uint32_t)dims[0], nRows = (uint32_t)nRows64;
  auto *rec = reinterpret_cast<unsigned long long *>(d.scratch + kNaRec);
  auto *src = reinterpret_cast<uint32_t *>(d.scratch + kNaSrc);
  auto *rowCount = reinterpret_cast<uint32_t *>(d.scratch + kNaCounts);
  uint32_t *rowCursor = rowCount + nRows + 1;
  auto *rowStartS = reinterpret_cast<uint32_t *>(d.scratch + kNaRowStart);
  auto *longRows = reinterpret_cast<uint32_t *>(d.scratch + kNaLong);
  auto *longCount = reinterpret_cast<uint32_t *>(d.scratch + kNaMisc);
  auto *status = reinterpret_cast<unsigned *>(d.scratch + kNaMisc + 4);
  auto *s1 = reinterpret_cast<uint32_t *>(d.scratch + kNaScan);
  uint32_t *s1x = s1 + kNaScanBlocks + 1, *s2 = s1x + kNaScanBlocks + 1;

  // every enqueue is checked where it is made; on a failure the stream is
  // drained before returning, so that no copy of this call is still running
  cudaError_t e = cudaSuccess;
  auto ok = [&](cudaError_t r) {
    if (e == cudaSuccess && r != cudaSuccess) e = r;
    return e == cudaSuccess;
  };
  ok(cudaMemsetAsync(rowCount, 0, 2 * ((size_t)nRows + 1) * sizeof(uint32_t), s));
  ok(cudaMemsetAsync(longCount, 0, 2 * sizeof(uint32_t), s));  // longCount and status
  if (e == cudaSuccess && n) {
    const int gridN = blocksFor(n, kBucketThreads);
    k_na_count<<<gridN, kBucketThreads, 0, s>>>(keys, (int)n, nx, nRows, rowCount, status);
    ok(cudaGetLastError());
  }
  const size_t count = (size_t)nRows + 1;
  const int nb1 = blocksFor(count, kScanBlock);
  if (e == cudaSuccess) {
    k_scan_blocks<<<nb1, kScanBlock, 0, s>>>(rowCount, (int)count, rowStartS, s1);
    ok(cudaGetLastError());
  }
  if (e == cudaSuccess && nb1 > 1) {
    k_scan_blocks<<<1, kScanBlock, 0, s>>>(s1, nb1, s1x, s2);
    if (ok(cudaGetLastError())) {
      k_scan_add<<<nb1, kScanBlock, 0, s>>>(rowStartS, (int)count, s1x);
      ok(cudaGetLastError());
    }
  }
  if (e == cudaSuccess && n) {
    const int gridN = blocksFor(n, kBucketThreads);
    k_na_scatter<<<gridN, kBucketThreads, 0, s>>>(keys, (int)n, nx, nRows, rowStartS, rowCursor, rec, src, status);
    if (ok(cudaGetLastError())) {
      const int smallBlocks = std::min(blocksFor((size_t)nRows * 32, kBucketThreads), 64 * d.sms);
      k_bucket_sort_small<<<smallBlocks, kBucketThreads, 0, s>>>(rowStartS, nRows, nx, rec, src, sortedKeys, order,
                                                                 longRows, longCount, nullptr);
    }
    if (ok(cudaGetLastError())) {
      k_bucket_sort_large<<<2 * d.sms, kBucketThreads, kLargeRow * 12, s>>>(
          rowStartS, nx, rec, src, sortedKeys, order, longRows, longCount, nullptr,
          DenseBin{nullptr, nullptr, 0, 0, nullptr});
      ok(cudaGetLastError());
    }
  }
  if (e == cudaSuccess && rowStart)
    ok(cudaMemcpyAsync(rowStart, rowStartS, count * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
  unsigned hostStatus = 0;
  if (e == cudaSuccess) ok(cudaMemcpyAsync(&hostStatus, status, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  const cudaError_t es = cudaStreamSynchronize(s);  // also on a failure: nothing of this call left running
  ok(es);
  if (e != cudaSuccess) {
    cudaGetLastError();
    naMessage(errMsg, errMsgCap, cudaGetErrorString(e));
    return LADDS_ERR_CUDA;
  }
  if (hostStatus & 1u) {
    naMessage(errMsg, errMsgCap, "invalid argument: a key lies beyond the grid (key >= dims[0]*dims[1]*dims[2])");
    return LADDS_ERR_INVALID_ARG;
  }
  if (hostStatus) {
    naMessage(errMsg, errMsgCap, "device check: inconsistent row counts");
    return LADDS_ERR_DEVICE_CHECK;
  }
  return LADDS_OK;
}

}  // extern "C"
