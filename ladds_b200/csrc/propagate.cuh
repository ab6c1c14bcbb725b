// propagate.cuh -- Yoshida-4 propagation kernel (+ fused cell-key output).
//
// Replaces YoshidaIntegrator::integrate(false) (called at Simulation.cpp:297;
// the integrator itself is in the non-vendored OrbitPropagator).  Form: DKD
// composition of Yoshida (1990): drift c1, kick d1, drift c2, kick d2,
// drift c2, kick d1, drift c1 -- three force evaluations per step at the
// stage times t + c1 dt, t + (c1+c2) dt, t + (c1+2 c2) dt.
//
// One thread per object, state held in registers across `nSteps` steps, so
// a multi-step launch touches HBM once (read 64 B + write 48 B per object).
// Ephemeris entries of all stages of the launch live in __constant__ memory
// (uniform across the warp).  The atmosphere table is staged in shared memory
// (the band index diverges across the warp).
#pragma once
#include "bulk_copy.cuh"
#include "cell_sort.cuh"
#include "forces.cuh"
#include "state.cuh"

namespace ladds {

constexpr int kMaxEphSteps = 128;  // 3 * 128 entries * 160 B = 61 KB of constant memory
__constant__ EphEntry c_eph[3 * kMaxEphSteps];
__constant__ AtmRow c_atm[kAtmBands] = LADDS_ATM_TABLE;

struct PropConsts {
  double hc1, hc2, hd1, hd2;  // Yoshida coefficients * dt
  uint32_t mask;
};

__device__ __forceinline__ uint32_t cellCoord(double v, double lo, double inv, int32_t n) {
  // floor((v - lo) * inv) with exactly these two roundings; NaN -> 0; clamped
  const double u = floor(__dmul_rn(__dsub_rn(v, lo), inv));
  if (!(u >= 0.0)) return 0u;
  if (u >= (double)n) return (uint32_t)(n - 1);
  return (uint32_t)u;
}

__device__ __forceinline__ uint32_t cellKey(double x, double y, double z, const GridDesc &g) {
  const uint32_t ix = cellCoord(x, g.boxMin[0], g.invCell, g.n[0]);
  const uint32_t iy = cellCoord(y, g.boxMin[1], g.invCell, g.n[1]);
  const uint32_t iz = cellCoord(z, g.boxMin[2], g.invCell, g.n[2]);
  return (iz * (uint32_t)g.n[1] + iy) * (uint32_t)g.n[0] + ix;
}

// nSteps Yoshida-4 steps of one object (stage ephemerides c_eph[ephBase ...]);
// a non-finite end state sets bit 1 of *status
template <bool SPLIT>
__device__ __forceinline__ void yoshidaSteps(double r[3], double v[3], double aom, double bc, uint32_t tag,
                                             int nSteps, int ephBase, const PropConsts &pc, const AtmShared &atm,
                                             unsigned *__restrict__ status) {
  uint32_t mask = pc.mask;
  if (tagAct(tag) == kEvasivePreserving) mask &= kPropKEP;  // Particle.h:48-52: Keplerian forces only
  double a[3];
  for (int st = 0; st < nSteps; ++st) {
    const EphEntry *e = &c_eph[ephBase + 3 * st];
#pragma unroll
    for (int k = 0; k < 3; ++k) r[k] += pc.hc1 * v[k];
    accel<SPLIT>(mask, r, v, aom, bc, e[0], atm, a);
#pragma unroll
    for (int k = 0; k < 3; ++k) v[k] += pc.hd1 * a[k];
#pragma unroll
    for (int k = 0; k < 3; ++k) r[k] += pc.hc2 * v[k];
    accel<SPLIT>(mask, r, v, aom, bc, e[1], atm, a);
#pragma unroll
    for (int k = 0; k < 3; ++k) v[k] += pc.hd2 * a[k];
#pragma unroll
    for (int k = 0; k < 3; ++k) r[k] += pc.hc2 * v[k];
    accel<SPLIT>(mask, r, v, aom, bc, e[2], atm, a);
#pragma unroll
    for (int k = 0; k < 3; ++k) v[k] += pc.hd1 * a[k];
#pragma unroll
    for (int k = 0; k < 3; ++k) r[k] += pc.hc1 * v[k];
  }
  if (!(isfinite(r[0]) && isfinite(r[1]) && isfinite(r[2]) && isfinite(v[0]) && isfinite(v[1]) && isfinite(v[2])))
    atomicOr(status, 1u);
}

// KEYS: also writes the cell key of the end position and counts it into its
// cell row (rowCount, arrival: see countRowArrival).
template <bool SPLIT, bool KEYS>
__global__ void __launch_bounds__(256, 4) k_propagate(DevState s, int n, int nSteps, int ephBase, PropConsts pc,
                                                   GridDesc g, uint32_t *__restrict__ keys,
                                                   uint32_t *__restrict__ rowCount, uint32_t *__restrict__ arrival,
                                                   unsigned *__restrict__ status) {
  __shared__ AtmShared atm;
  loadAtmTable(atm, c_atm);
  __syncthreads();
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (!KEYS && j >= n) return;
  const bool inRange = j < n;
  const uint32_t tag = inRange ? s.tag[j] : kTagDummy;
  double r[3] = {0.0, 0.0, 0.0};
  if (inRange) {
    r[0] = s.x[j];
    r[1] = s.y[j];
    r[2] = s.z[j];
  }
  if (!tagDummy(tag)) {
    double v[3] = {s.vx[j], s.vy[j], s.vz[j]};
    const double aom = s.aom[j], bc = s.bc[j];
    yoshidaSteps<SPLIT>(r, v, aom, bc, tag, nSteps, ephBase, pc, atm, status);
    s.x[j] = r[0];
    s.y[j] = r[1];
    s.z[j] = r[2];
    s.vx[j] = v[0];
    s.vy[j] = v[1];
    s.vz[j] = v[2];
  }
  if (KEYS) {  // every lane of the warp reaches this point
    const uint32_t key = cellKey(r[0], r[1], r[2], g);
    const uint32_t a = countRowArrival(key, inRange, (uint32_t)g.n[0], rowCount);
    if (inRange) {
      keys[j] = key;
      arrival[j] = a;
    }
  }
}

// The per-scan propagation (with cell keys) over a persistent grid.  CTA b
// takes the tiles b, b + gridDim.x, ... of kStageObjects consecutive objects.
// While a tile is propagated, the state of the CTA's next tile is already on
// its way into shared memory: one thread issues nine bulk copies (x, y, z, vx,
// vy, vz, aom, bc: 2 KB each; tags: 1 KB) completed on an mbarrier, so no
// warp stalls on its loads after the first tile, and the atmosphere table is
// staged once per CTA instead of once per 256 objects.  The partial tile at
// the end (n % kStageObjects objects) is read directly.  Results are those of
// k_propagate<SPLIT, true> bit for bit (same per-object arithmetic).  A wait
// that runs out (it cannot, unless a copy is lost) sets bit 8 of *status.
constexpr int kStageObjects = 256;
constexpr int kStageArrays = 8;
constexpr uint32_t kStageTxBytes = kStageArrays * kStageObjects * 8 + kStageObjects * 4;
constexpr uint32_t kStageWaitPolls = 1u << 22;

template <bool SPLIT>
__global__ void __launch_bounds__(kStageObjects, 4) k_propagate_staged(DevState s, int n, int nSteps, int ephBase,
                                                                      PropConsts pc, GridDesc g,
                                                                      uint32_t *__restrict__ keys,
                                                                      uint32_t *__restrict__ rowCount,
                                                                      uint32_t *__restrict__ arrival,
                                                                      unsigned *__restrict__ status) {
  __shared__ AtmShared atm;
  __shared__ __align__(16) double sv[kStageArrays][kStageObjects];
  __shared__ __align__(16) uint32_t stag[kStageObjects];
  __shared__ __align__(8) unsigned long long sbar;
  const int tid = threadIdx.x;
  const int nFull = n / kStageObjects, nTiles = (n + kStageObjects - 1) / kStageObjects;
  // one thread: the copies of full tile t into the stage
  auto issue = [&](int t) {
    const size_t base = (size_t)t * kStageObjects;
    const double *src[kStageArrays] = {s.x, s.y, s.z, s.vx, s.vy, s.vz, s.aom, s.bc};
    asyncProxyFence();
    mbarArriveExpectTx(&sbar, kStageTxBytes);
#pragma unroll
    for (int a = 0; a < kStageArrays; ++a) bulkLoad(sv[a], src[a] + base, kStageObjects * 8, &sbar);
    bulkLoad(stag, s.tag + base, kStageObjects * 4, &sbar);
  };
  if (tid == 0) {
    mbarInit(&sbar, 1);
    mbarInitFence();
  }
  loadAtmTable(atm, c_atm);
  __syncthreads();
  int t = blockIdx.x;
  if (tid == 0 && t < nFull) issue(t);
  for (uint32_t it = 0; t < nTiles; t += gridDim.x) {  // t is the same in every thread of the CTA
    const int j = t * kStageObjects + tid;
    const bool inRange = j < n;
    double r[3] = {0.0, 0.0, 0.0}, v[3] = {0.0, 0.0, 0.0}, aom = 0.0, bc = 0.0;
    uint32_t tag = kTagDummy;
    if (t < nFull) {
      if (!mbarWait(&sbar, it & 1u, kStageWaitPolls)) atomicOr(status, 8u);
      ++it;
      r[0] = sv[0][tid];
      r[1] = sv[1][tid];
      r[2] = sv[2][tid];
      v[0] = sv[3][tid];
      v[1] = sv[4][tid];
      v[2] = sv[5][tid];
      aom = sv[6][tid];
      bc = sv[7][tid];
      tag = stag[tid];
      __syncthreads();  // the stage is free: the next tile's copies go out now
      if (tid == 0 && t + (int)gridDim.x < nFull) issue(t + (int)gridDim.x);
    } else if (inRange) {
      tag = s.tag[j];
      r[0] = s.x[j];
      r[1] = s.y[j];
      r[2] = s.z[j];
      v[0] = s.vx[j];
      v[1] = s.vy[j];
      v[2] = s.vz[j];
      aom = s.aom[j];
      bc = s.bc[j];
    }
    if (!tagDummy(tag)) {
      yoshidaSteps<SPLIT>(r, v, aom, bc, tag, nSteps, ephBase, pc, atm, status);
      s.x[j] = r[0];
      s.y[j] = r[1];
      s.z[j] = r[2];
      s.vx[j] = v[0];
      s.vy[j] = v[1];
      s.vz[j] = v[2];
    }
    // every lane of the warp reaches this point
    const uint32_t key = cellKey(r[0], r[1], r[2], g);
    const uint32_t a = countRowArrival(key, inRange, (uint32_t)g.n[0], rowCount);
    if (inRange) {
      keys[j] = key;
      arrival[j] = a;
    }
  }
}

// slots of the live objects whose cell layer iz (the z index of the cell key)
// lies in [lo, hi), appended in any order
__global__ void k_select_layers(const double *__restrict__ z, const uint32_t *__restrict__ tag, int n, GridDesc g,
                                int32_t lo, int32_t hi, uint32_t *__restrict__ out, unsigned *__restrict__ count,
                                unsigned cap) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n || tagDummy(tag[j])) return;
  const int32_t iz = (int32_t)cellCoord(z[j], g.boxMin[2], g.invCell, g.n[2]);
  if (iz < lo || iz >= hi) return;
  const unsigned q = atomicAdd(count, 1u);
  if (q < cap) out[q] = tagSlot(tag[j]);
}

// live objects per cell layer
__global__ void k_layer_histogram(const double *__restrict__ z, const uint32_t *__restrict__ tag, int n, GridDesc g,
                                  unsigned long long *__restrict__ counts) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n || tagDummy(tag[j])) return;
  atomicAdd(&counts[cellCoord(z[j], g.boxMin[2], g.invCell, g.n[2])], 1ull);
}

// Ephemeris of the stage times of `nSteps` steps starting at iteration `iter`
// (one thread per stage), written to a global staging table that the host then
// copies into c_eph.
__global__ void k_ephemeris(EphEntry *__restrict__ out, int nSteps, int64_t iter, double t0, double dt, double hc1,
                            double hc2, double jdEpoch, double theta0) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 3 * nSteps) return;
  const int st = i / 3, stage = i % 3;
  const double tn = t0 + (double)(iter + st) * dt;
  double tau = tn + hc1;
  if (stage >= 1) tau += hc2;
  if (stage >= 2) tau += hc2;
  ephemeris(jdEpoch, theta0, tau, out[i]);
}

// cell keys of the current positions + their row counts (as k_propagate<*, true>)
__global__ void k_cell_keys(const double *__restrict__ x, const double *__restrict__ y, const double *__restrict__ z,
                            int n, GridDesc g, uint32_t *__restrict__ keys, uint32_t *__restrict__ rowCount,
                            uint32_t *__restrict__ arrival) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const bool inRange = j < n;
  const uint32_t key = inRange ? cellKey(x[j], y[j], z[j], g) : 0u;
  const uint32_t a = countRowArrival(key, inRange, (uint32_t)g.n[0], rowCount);
  if (inRange) {
    keys[j] = key;
    arrival[j] = a;
  }
}

}  // namespace ladds
