// pair_scan.cuh -- two-phase pair scan over the cell-sorted population.
//
// Phase 1, k_pair_candidates: one thread per object of the cell order walks
// its half-shell like a Newton3 linked-cell traversal -- the rest of its own
// row window (ix .. ix+R, later objects only) and the rows (dz,dy) > (0,0),
// each window ix-R .. ix+R.  A window is located with two reads of the row's
// cell-offset table (written by the cell sort) instead of a search; rows whose
// offsets do not fit 16 bits, or grids too large for the table, fall back to a
// binary search on the sorted keys.  A binary32 distance test with a margin
// larger than its rounding error rejects most candidates; the survivors get
// the exact binary64 cutoff gate d^2 <= cutoff^2 (CollisionFunctor.cpp:71-77,
// same rounding) or its near band.  Candidates are buffered per warp in shared
// memory and appended with one global atomic per warp (no block barriers).
//
// Phase 2, k_pair_eval: one thread per candidate evaluates the functor
// (CollisionFunctor.cpp:40-131) and appends the records.
#pragma once
#include <cooperative_groups.h>

#include "conjunction.cuh"

namespace ladds {

namespace cg = cooperative_groups;

constexpr int kScanCta = 128;
constexpr int kWarpCand = 128;  // candidates buffered per warp before a global append

// Direct global append (only for candidates beyond a warp's shared buffer).
__device__ __forceinline__ void appendCandidateGlobal(uint32_t a, uint32_t b, uint2 *__restrict__ cand,
                                                      unsigned long long *__restrict__ count,
                                                      unsigned long long cap) {
  cg::coalesced_group grp = cg::coalesced_threads();
  unsigned long long base = 0;
  if (grp.thread_rank() == 0) base = atomicAdd(count, (unsigned long long)grp.size());
  base = grp.shfl(base, 0);
  const unsigned long long pos = base + grp.thread_rank();
  if (pos < cap) cand[pos] = make_uint2(a, b);
}

// [lo, hi) of the cells xlo..xhi of row r2 in the sorted arrays
__device__ __forceinline__ void rowWindow(uint32_t r2, uint32_t xlo, uint32_t xhi, uint32_t nx,
                                          const uint32_t *__restrict__ rowStart,
                                          const uint16_t *__restrict__ cellOff,
                                          const uint32_t *__restrict__ skeys, uint32_t &lo, uint32_t &hi) {
  const uint32_t rs0 = __ldg(&rowStart[r2]), rs1 = __ldg(&rowStart[r2 + 1]);
  if (rs1 == rs0) {
    lo = hi = rs0;
    return;
  }
  if (cellOff && rs1 - rs0 <= 65535u) {
    const uint16_t *t = cellOff + (size_t)r2 * cellOffPitch(nx);
    lo = rs0 + __ldg(&t[xlo]);
    hi = rs0 + __ldg(&t[xhi + 1]);
  } else {
    const uint32_t rowBase = r2 * nx;
    lo = lowerBound(skeys, rs0, rs1, rowBase + xlo);
    hi = lowerBound(skeys, lo, rs1, rowBase + xhi + 1);
  }
}

// Binary32 pre-filter and exact binary64 gate of one candidate pair (j, k)
// with its positions already loaded; survivors go to the warp's buffer.
__device__ __forceinline__ void testCandidate(uint32_t j, uint32_t k, float4 mf, float4 q,
                                              const double4 *__restrict__ pos4, double cutoffSq, double nearRel,
                                              float cutF, uint2 *sCandW, uint32_t *sNW, uint2 *__restrict__ cand,
                                              unsigned long long *__restrict__ candCount,
                                              unsigned long long candCap) {
  const float dx = mf.x - q.x, dy = mf.y - q.y, dz = mf.z - q.z;
  const float lim = cutF + 2.0f * (mf.w + q.w);
  if (dx * dx + dy * dy + dz * dz > lim * lim * 1.000001f) return;
  const double4 me = pos4[j], o = pos4[k];
  double d[3];
  d[0] = __dsub_rn(me.x, o.x);
  d[1] = __dsub_rn(me.y, o.y);
  d[2] = __dsub_rn(me.z, o.z);
  const double d2 = dot3rn(d, d);
  if (d2 > cutoffSq && !nearBand(d2, cutoffSq, nearRel)) return;
  const uint32_t slot = atomicAdd(sNW, 1u);  // shared counter: no global contention
  if (slot < (uint32_t)kWarpCand)
    sCandW[slot] = make_uint2(j, k);
  else
    appendCandidateGlobal(j, k, cand, candCount, candCap);
}

// owner lane of item t: the largest lane whose excl <= t (lanes with empty
// windows share the next lane's excl, so the largest is the one that owns t)
__device__ __forceinline__ int windowOwner(uint32_t excl, uint32_t item) {
  int owner = 0;
#pragma unroll
  for (int step = 16; step >= 1; step >>= 1) {
    const uint32_t e = __shfl_sync(0xffffffffu, excl, owner + step);
    if (e <= item) owner += step;
  }
  return owner;
}

// Warp-balanced walk of one neighbour row: lane l owns the window [lo, hi) of
// its object; the windows of the warp are concatenated (exclusive prefix
// `excl`) and dealt out 32 items per round, so every lane tests one pair per
// round however uneven the windows are.
__device__ __forceinline__ void warpWindowPairs(uint32_t lo, uint32_t hi, int lane, int warpBase,
                                                const double4 *__restrict__ pos4, const float4 *__restrict__ posf,
                                                double cutoffSq, double nearRel, float cutF, uint2 *sCandW,
                                                uint32_t *sNW, uint2 *__restrict__ cand,
                                                unsigned long long *__restrict__ candCount,
                                                unsigned long long candCap) {
  const uint32_t cnt = hi - lo;
  uint32_t incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
  const uint32_t excl = incl - cnt;
  for (uint32_t base = 0; base < total; base += 32u) {
    const uint32_t item = base + (uint32_t)lane;
    const int owner = windowOwner(excl, item);
    const uint32_t oLo = __shfl_sync(0xffffffffu, lo, owner), oEx = __shfl_sync(0xffffffffu, excl, owner);
    if (item >= total) continue;
    const uint32_t jj = (uint32_t)(warpBase + owner), k = oLo + (item - oEx);
    testCandidate(jj, k, __ldg(&posf[jj]), __ldg(&posf[k]), pos4, cutoffSq, nearRel, cutF, sCandW, sNW, cand,
                  candCount, candCap);
  }
}

// cutF: cutoff * (1 + nearRel) rounded up, so that every pair the exact gate or
// its near band accepts passes the binary32 test.  The loops over the
// neighbour rows are warp-uniform; inactive lanes contribute empty windows.
__global__ void __launch_bounds__(kScanCta) k_pair_candidates(const uint32_t *__restrict__ tags,
                                                              const double4 *__restrict__ pos4,
                                                              const float4 *__restrict__ posf, int n,
                                                              const uint32_t *__restrict__ skeys,
                                                              const uint32_t *__restrict__ rowStart,
                                                              const uint16_t *__restrict__ cellOff, GridDesc g,
                                                              double cutoffSq, double nearRel, float cutF,
                                                              uint2 *__restrict__ cand,
                                                              unsigned long long *__restrict__ candCount,
                                                              unsigned long long candCap) {
  __shared__ uint2 sCand[kScanCta / 32][kWarpCand];
  __shared__ uint32_t sN[kScanCta / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) sN[warp] = 0;
  __syncwarp();
  const int warpBase = blockIdx.x * kScanCta + warp * 32;
  const int j = warpBase + lane;
  const bool inRange = j < n;
  const uint32_t myTag = inRange ? tags[j] : kTagDummy;
  const bool active = inRange && !tagDummy(myTag);
  const int32_t nx = g.n[0], ny = g.n[1], nz = g.n[2], R = g.reach;
  int32_t ix = 0, iy = 0, iz = 0;
  if (active) {
    const uint32_t key = skeys[j];
    ix = (int32_t)(key % (uint32_t)nx);
    const uint32_t row = key / (uint32_t)nx;
    iy = (int32_t)(row % (uint32_t)ny);
    iz = (int32_t)(row / (uint32_t)ny);
  }
  const uint32_t xlo = (uint32_t)max(ix - R, 0), xhi = (uint32_t)min(ix + R, nx - 1);
  for (int dz = 0; dz <= R; ++dz) {
    for (int dy = (dz == 0 ? 0 : -R); dy <= R; ++dy) {
      const int32_t jz = iz + dz, jy = iy + dy;
      uint32_t lo = 0, hi = 0;
      if (active && jz < nz && jy >= 0 && jy < ny) {
        const uint32_t r2 = (uint32_t)jz * (uint32_t)ny + (uint32_t)jy;
        if (dz == 0 && dy == 0) {
          uint32_t l0;
          rowWindow(r2, (uint32_t)ix, xhi, (uint32_t)nx, rowStart, cellOff, skeys, l0, hi);
          lo = (uint32_t)j + 1u;  // own cell: later objects only
          if (hi < lo) hi = lo;
        } else {
          rowWindow(r2, xlo, xhi, (uint32_t)nx, rowStart, cellOff, skeys, lo, hi);
        }
      }
      warpWindowPairs(lo, hi, lane, warpBase, pos4, posf, cutoffSq, nearRel, cutF, sCand[warp], &sN[warp], cand,
                      candCount, candCap);
    }
  }
  // one global append per warp for its buffered candidates
  __syncwarp();
  const uint32_t m = min(sN[warp], (uint32_t)kWarpCand);
  unsigned long long base = 0;
  if (lane == 0 && m) base = atomicAdd(candCount, (unsigned long long)m);
  base = __shfl_sync(0xffffffffu, base, 0);
  for (uint32_t i = lane; i < m; i += 32) {
    const unsigned long long pos = base + i;
    if (pos < candCap) cand[pos] = sCand[warp][i];
  }
}

// grid-stride over the candidates (count read on the device)
__global__ void __launch_bounds__(256) k_pair_eval(ScanPack pk, const uint2 *__restrict__ cand,
                                                   const unsigned long long *__restrict__ candCount,
                                                   unsigned long long candCap,
                                                   unsigned long long *__restrict__ candNeed, ScanConsts c,
                                                   const int64_t *__restrict__ iterPtr, int64_t iterOffset,
                                                   ladds_pair *__restrict__ out,
                                                   unsigned long long *__restrict__ count, unsigned long long cap) {
  const unsigned long long total = *candCount;
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicMax(candNeed, total);
  const unsigned long long m = total < candCap ? total : candCap;
  const int64_t it = *iterPtr + iterOffset;  // iteration index stored in the records
  const uint32_t step = it < 0 ? 0u : (uint32_t)it;
  for (unsigned long long q = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; q < m;
       q += (unsigned long long)gridDim.x * blockDim.x) {
    const uint2 p = cand[q];
    Obj a, b;
    loadObjPacked(pk, p.x, a);
    loadObjPacked(pk, p.y, b);
    if (tagDummy(a.tag) || tagDummy(b.tag)) continue;
    double d[3];
    d[0] = __dsub_rn(a.r[0], b.r[0]);
    d[1] = __dsub_rn(a.r[1], b.r[1]);
    d[2] = __dsub_rn(a.r[2], b.r[2]);
    const double d2 = dot3rn(d, d);
    const bool aFirst = a.id < b.id || (a.id == b.id && tagSlot(a.tag) < tagSlot(b.tag));
    const Obj &I = aFirst ? a : b;
    const Obj &J = aFirst ? b : a;
    double dl2 = 0.0, point[3] = {0.0, 0.0, 0.0};
    const uint32_t f = functorPair(c, I, J, d2, dl2, point);
    if (f) emitPair(I, J, dl2, point, f, step, out, count, cap);
  }
}

// Explicit pair list: one thread per (first[k], second[k]).
__global__ void __launch_bounds__(256) k_functor_pairs(const ladds_object *__restrict__ first,
                                                       const ladds_object *__restrict__ second, int nPairs,
                                                       ScanConsts c, ladds_pair *__restrict__ out,
                                                       unsigned long long *__restrict__ count,
                                                       unsigned long long cap) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nPairs) return;
  Obj a, b;
  const ladds_object *src[2] = {&first[q], &second[q]};
  Obj *dst[2] = {&a, &b};
#pragma unroll
  for (int w = 0; w < 2; ++w) {
    const ladds_object &o = *src[w];
    for (int k = 0; k < 3; ++k) {
      dst[w]->r[k] = o.r[k];
      dst[w]->v[k] = o.v[k];
    }
    dst[w]->radius = o.radius;
    dst[w]->id = o.id;
    dst[w]->parent = o.parentId;
    dst[w]->tag = makeTag(o.slot, o.activity, false);
  }
  double d[3];
  d[0] = __dsub_rn(a.r[0], b.r[0]);
  d[1] = __dsub_rn(a.r[1], b.r[1]);
  d[2] = __dsub_rn(a.r[2], b.r[2]);
  const double d2 = dot3rn(d, d);
  const bool aFirst = a.id < b.id || (a.id == b.id && tagSlot(a.tag) < tagSlot(b.tag));
  const Obj &I = aFirst ? a : b;
  const Obj &J = aFirst ? b : a;
  double dl2 = 0.0, point[3] = {0.0, 0.0, 0.0};
  const uint32_t f = functorPair(c, I, J, d2, dl2, point);
  if (f) emitPair(I, J, dl2, point, f, 0u, out, count, cap);
}

}  // namespace ladds
