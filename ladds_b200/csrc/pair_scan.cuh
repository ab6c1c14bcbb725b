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
    const uint16_t *t = cellOff + (size_t)r2 * (nx + 1);
    lo = rs0 + __ldg(&t[xlo]);
    hi = rs0 + __ldg(&t[xhi + 1]);
  } else {
    const uint32_t rowBase = r2 * nx;
    lo = lowerBound(skeys, rs0, rs1, rowBase + xlo);
    hi = lowerBound(skeys, lo, rs1, rowBase + xhi + 1);
  }
}

// cutF: cutoff * (1 + nearRel) rounded up, so that every pair the exact gate or
// its near band accepts passes the binary32 test.
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
  const int j = blockIdx.x * kScanCta + (int)threadIdx.x;
  const bool inRange = j < n;
  const uint32_t myTag = inRange ? tags[j] : kTagDummy;
  const bool active = inRange && !tagDummy(myTag);
  if (active) {
    const int32_t nx = g.n[0], ny = g.n[1], nz = g.n[2], R = g.reach;
    const uint32_t key = skeys[j];
    const double4 me = pos4[j];
    const float4 mf = posf[j];
    const int32_t ix = (int32_t)(key % (uint32_t)nx);
    const uint32_t row = key / (uint32_t)nx;
    const int32_t iy = (int32_t)(row % (uint32_t)ny), iz = (int32_t)(row / (uint32_t)ny);
    const uint32_t xlo = (uint32_t)max(ix - R, 0), xhi = (uint32_t)min(ix + R, nx - 1);
    for (int dz = 0; dz <= R; ++dz) {
      const int32_t jz = iz + dz;
      if (jz >= nz) break;
      for (int dy = (dz == 0 ? 0 : -R); dy <= R; ++dy) {
        const int32_t jy = iy + dy;
        if (jy < 0 || jy >= ny) continue;
        const uint32_t r2 = (uint32_t)jz * (uint32_t)ny + (uint32_t)jy;
        uint32_t lo, hi;
        if (dz == 0 && dy == 0) {
          uint32_t l0;
          rowWindow(r2, (uint32_t)ix, xhi, (uint32_t)nx, rowStart, cellOff, skeys, l0, hi);
          lo = (uint32_t)j + 1u;  // own cell: later objects only
        } else {
          rowWindow(r2, xlo, xhi, (uint32_t)nx, rowStart, cellOff, skeys, lo, hi);
        }
        for (uint32_t k = lo; k < hi; ++k) {
          const float4 q = __ldg(&posf[k]);
          const float dx = mf.x - q.x, dy2 = mf.y - q.y, dz2 = mf.z - q.z;
          const float lim = cutF + 2.0f * (mf.w + q.w);
          if (dx * dx + dy2 * dy2 + dz2 * dz2 > lim * lim * 1.000001f) continue;
          const double4 o = pos4[k];
          double d[3];
          d[0] = __dsub_rn(me.x, o.x);
          d[1] = __dsub_rn(me.y, o.y);
          d[2] = __dsub_rn(me.z, o.z);
          const double d2 = dot3rn(d, d);
          if (d2 > cutoffSq && !nearBand(d2, cutoffSq, nearRel)) continue;
          const uint32_t slot = atomicAdd(&sN[warp], 1u);  // shared counter: no global contention
          if (slot < (uint32_t)kWarpCand)
            sCand[warp][slot] = make_uint2((uint32_t)j, k);
          else
            appendCandidateGlobal((uint32_t)j, k, cand, candCount, candCap);
        }
      }
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
