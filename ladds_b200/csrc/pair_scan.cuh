// pair_scan.cuh -- two-phase pair scan over the cell-sorted population.
//
// Phase 1, k_pair_candidates: a CTA takes kScanCta consecutive objects of the
// cell order.  Their neighbour rows form R+1 contiguous runs of the sorted
// arrays: rows [rFirst, rLast+R] of the own plane and, for every dz in 1..R,
// rows [rFirst + dz*ny - R, rLast + dz*ny + R] (rows are numbered iz*ny + iy,
// so the rows of a plane are contiguous and so are their objects).  Those runs
// (keys + binary32 positions with a rounding bound) and their row-start
// entries are staged in shared memory; each thread then walks its half-shell
// -- the rest of its own row window and the rows (dz,dy) > (0,0) -- with
// binary searches that only touch shared memory.  A binary32 distance test
// with a margin larger than its rounding error rejects most candidates; the
// survivors get the exact binary64 cutoff gate d^2 <= cutoff^2
// (CollisionFunctor.cpp:71-77, same rounding) or its near band, are buffered
// per CTA and appended to the candidate list with one global atomic per CTA.
// When a run does not fit the stage, the CTA reads it from global memory.
//
// Phase 2, k_pair_eval: one thread per candidate evaluates the functor
// (CollisionFunctor.cpp:40-131) and appends the records.
#pragma once
#include <cooperative_groups.h>

#include "conjunction.cuh"

namespace ladds {

namespace cg = cooperative_groups;

constexpr int kScanCta = 256;
constexpr int kStageMax = 1280;   // staged objects per CTA (25 KB of shared memory)
constexpr int kCandStage = 2048;  // candidates buffered per CTA before one global append (16 KB)
constexpr int kMaxStagedRuns = 9; // reach <= 8
constexpr int kRowStage = 63;     // staged row-start entries per run (rows of the run + 1)

// Direct global append (only for candidates beyond a CTA's shared buffer).
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

// cutF: cutoff * (1 + nearRel) rounded up, so that every pair the exact gate or
// its near band accepts passes the binary32 test.
__global__ void __launch_bounds__(kScanCta) k_pair_candidates(const uint32_t *__restrict__ tags,
                                                              const double4 *__restrict__ pos4,
                                                              const float4 *__restrict__ posf, int n,
                                                              const uint32_t *__restrict__ skeys,
                                                              const uint32_t *__restrict__ rowStart, GridDesc g,
                                                              double cutoffSq, double nearRel, float cutF,
                                                              uint2 *__restrict__ cand,
                                                              unsigned long long *__restrict__ candCount,
                                                              unsigned long long candCap) {
  __shared__ uint32_t sKeys[kStageMax];
  __shared__ float4 sPos[kStageMax];
  __shared__ uint2 sCand[kCandStage];
  __shared__ uint32_t sRow[kMaxStagedRuns][kRowStage + 1];
  __shared__ int64_t sRowA[kMaxStagedRuns];   // first row of each run
  __shared__ uint32_t sRowN[kMaxStagedRuns];  // rows of each run (0: run empty)
  __shared__ uint32_t sBase[kMaxStagedRuns], sCnt[kMaxStagedRuns], sOff[kMaxStagedRuns + 1];
  __shared__ int sStaged;
  __shared__ uint32_t sCandN;
  __shared__ unsigned long long sCandBase;
  const int s0 = blockIdx.x * kScanCta;
  if (s0 >= n) return;  // uniform over the CTA
  const int32_t nx = g.n[0], ny = g.n[1], nz = g.n[2], R = g.reach;
  const int64_t nRows = (int64_t)ny * nz;
  // own object, loaded before the set-up barrier
  const int j = s0 + (int)threadIdx.x;
  const bool inRange = j < n;
  const uint32_t myTag = inRange ? tags[j] : kTagDummy;
  const uint32_t key = inRange ? skeys[j] : 0u;
  const double4 me = inRange ? pos4[j] : make_double4(0.0, 0.0, 0.0, 0.0);
  const float4 mf = inRange ? posf[j] : make_float4(0.f, 0.f, 0.f, 0.f);
  // set-up: thread d <= R owns run d
  if ((int)threadIdx.x <= R) {
    const int d = threadIdx.x;
    const int sLast = min(s0 + kScanCta, n) - 1;
    const int64_t rFirst = skeys[s0] / (uint32_t)nx, rLast = skeys[sLast] / (uint32_t)nx;
    int64_t a = d == 0 ? rFirst : rFirst + (int64_t)d * ny - R;
    int64_t b = d == 0 ? rLast + R : rLast + (int64_t)d * ny + R;
    a = max(a, (int64_t)0);
    b = min(b, nRows - 1);
    uint32_t p0 = 0, p1 = 0;
    if (a <= b) {
      p0 = rowStart[a];
      p1 = rowStart[b + 1];
    }
    sRowA[d] = a;
    sRowN[d] = a <= b ? (uint32_t)(b - a + 1) : 0u;
    sBase[d] = p0;
    sCnt[d] = p1 - p0;
    if (d == 0) sCandN = 0;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t total = 0;
    for (int d = 0; d <= R; ++d) {
      sOff[d] = total;
      total += sCnt[d];
    }
    sOff[R + 1] = total;
    sStaged = total <= (uint32_t)kStageMax;
  }
  // row-start entries of the runs (rows a .. a+rows, inclusive of the end entry)
  for (int d = 0; d <= R; ++d) {
    const uint32_t nr = sRowN[d];
    if (nr && nr <= (uint32_t)kRowStage)
      for (uint32_t i = threadIdx.x; i <= nr; i += kScanCta) sRow[d][i] = rowStart[sRowA[d] + i];
  }
  __syncthreads();
  const bool staged = sStaged != 0;
  if (staged) {
    for (int d = 0; d <= R; ++d) {
      const uint32_t cnt = sCnt[d], off = sOff[d], base = sBase[d];
      for (uint32_t i = threadIdx.x; i < cnt; i += kScanCta) {
        sKeys[off + i] = skeys[base + i];
        sPos[off + i] = posf[base + i];
      }
    }
  }
  __syncthreads();
  const bool active = inRange && !tagDummy(myTag);
  const int32_t ix = (int32_t)(key % (uint32_t)nx);
  const uint32_t row = key / (uint32_t)nx;
  const int32_t iy = (int32_t)(row % (uint32_t)ny), iz = (int32_t)(row / (uint32_t)ny);
  const uint32_t xlo = (uint32_t)max(ix - R, 0), xhi = (uint32_t)min(ix + R, nx - 1);
  for (int dz = 0; active && dz <= R; ++dz) {
    const int32_t jz = iz + dz;
    if (jz >= nz) break;
    const uint32_t *K = staged ? sKeys + sOff[dz] : skeys;
    const float4 *P = staged ? sPos + sOff[dz] : posf;
    const uint32_t base = staged ? sBase[dz] : 0u;
    const bool rowsStaged = sRowN[dz] <= (uint32_t)kRowStage;
    const int64_t rowA = sRowA[dz];
    for (int dy = (dz == 0 ? 0 : -R); dy <= R; ++dy) {
      const int32_t jy = iy + dy;
      if (jy < 0 || jy >= ny) continue;
      const uint32_t r2 = (uint32_t)jz * (uint32_t)ny + (uint32_t)jy;
      const uint32_t rowBase = r2 * (uint32_t)nx;
      uint32_t rs0, rs1;
      if (rowsStaged) {
        const uint32_t li = (uint32_t)((int64_t)r2 - rowA);
        rs0 = sRow[dz][li];
        rs1 = sRow[dz][li + 1];
      } else {
        rs0 = rowStart[r2];
        rs1 = rowStart[r2 + 1];
      }
      const uint32_t hi = rs1 - base;
      uint32_t k = (dz == 0 && dy == 0) ? (uint32_t)j + 1u - base : lowerBound(K, rs0 - base, hi, rowBase + xlo);
      const uint32_t hiKey = rowBase + xhi;
      for (; k < hi && K[k] <= hiKey; ++k) {
        const float4 q = P[k];
        const float dx = mf.x - q.x, dy2 = mf.y - q.y, dz2 = mf.z - q.z;
        const float lim = cutF + 2.0f * (mf.w + q.w);
        if (dx * dx + dy2 * dy2 + dz2 * dz2 > lim * lim * 1.000001f) continue;
        const double4 o = pos4[k + base];
        double d[3];
        d[0] = __dsub_rn(me.x, o.x);
        d[1] = __dsub_rn(me.y, o.y);
        d[2] = __dsub_rn(me.z, o.z);
        const double d2 = dot3rn(d, d);
        if (d2 > cutoffSq && !nearBand(d2, cutoffSq, nearRel)) continue;
        const uint32_t slot = atomicAdd(&sCandN, 1u);  // shared-memory counter: no global contention
        if (slot < (uint32_t)kCandStage)
          sCand[slot] = make_uint2((uint32_t)j, k + base);
        else
          appendCandidateGlobal((uint32_t)j, k + base, cand, candCount, candCap);
      }
    }
  }
  // one global append for the CTA's buffered candidates
  __syncthreads();
  const uint32_t m = min(sCandN, (uint32_t)kCandStage);
  if (threadIdx.x == 0) sCandBase = m ? atomicAdd(candCount, (unsigned long long)m) : 0ull;
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < m; i += kScanCta) {
    const unsigned long long pos = sCandBase + i;
    if (pos < candCap) cand[pos] = sCand[i];
  }
}

// grid-stride over the candidates (count read on the device)
__global__ void __launch_bounds__(256) k_pair_eval(DevState s, const uint2 *__restrict__ cand,
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
    loadObj(s, (int)p.x, a);
    loadObj(s, (int)p.y, b);
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

}  // namespace ladds
