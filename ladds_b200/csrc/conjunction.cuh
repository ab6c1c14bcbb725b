// conjunction.cuh -- cell table and pair scan.
//
// Replaces AutoPas::iteratePairwise(&CollisionFunctor) (Simulation.cpp:220,
// external traversal) together with CollisionFunctor::AoSFunctor
// (CollisionFunctor.cpp:40-131) and utils::distanceByLinearInterpolation
// (DistanceApproximation.cpp:13-58).
//
// After the radix sort the population is gathered into cell order.  Keys are
// row-major, (iz*ny + iy)*nx + ix, so the cells (ix-R..ix+R) of one row are a
// contiguous key window.  rowStart[r] = first sorted index of row r.  One
// thread per sorted object visits, like a Newton3 linked-cell traversal, each
// neighbouring pair once: the rest of its own row window (ix..ix+R, later
// objects only) and the rows (dz,dy) > (0,0) lexicographically, each located by
// a binary search inside its row.  The candidate test and the functor use
// explicitly rounded operations (__dmul_rn / __dadd_rn / __dsub_rn /
// __ddiv_rn) in the reference's evaluation order, so results are bit-identical
// to a binary64 CPU evaluation without FMA contraction, NaN path included.
#pragma once
#include <algorithm>
#include <cmath>

#include "../../include/ladds_gpu.h"
#include "physics.cuh"
#include "state.cuh"

namespace ladds {

// float copy of a position with a bound on its rounding error per coordinate
__device__ __forceinline__ float4 floatPosition(double x, double y, double z) {
  const double m = fmax(fabs(x), fmax(fabs(y), fabs(z)));
  return make_float4((float)x, (float)y, (float)z, (float)(m * 0x1p-22) + 1e-12f);
}

// What the pair scan reads of the cell-ordered population: binary32 copies
// (positions with their rounding bound, velocities with the radius rounded up)
// in cell order, and, for the few pairs that reach the binary64 functor, the
// state as it was before the gather (src, indexed through perm) -- the next
// propagation, which runs beside the scan, writes only the gathered copy.
// Breakup group of an object in the scan: its parent id when that fits 32
// bits, else kNoGroup (no parent, or an id too large to compare here: such
// pairs are left to the functor's own parent test).  Two objects of one group
// cannot yield a record (CollisionFunctor.cpp:64-67), so the pair scan skips
// them before they become candidates.
constexpr uint32_t kNoGroup = 0xffffffffu;
__device__ __forceinline__ uint32_t groupOf(uint64_t parent) {
  return parent < (uint64_t)kNoGroup ? (uint32_t)parent : kNoGroup;
}

struct ScanPack {
  float4 *posf;          // binary32 x, y, z + rounding bound
  float4 *velf;          // binary32 vx, vy, vz + radius rounded up
  DevState src;          // state before the gather
  const uint32_t *perm;  // cell-order position -> index in src
  uint32_t *grp;         // breakup group per cell-order position (null: no object has a parent)
};

__global__ void k_permute(DevState src, DevState dst, const uint32_t *__restrict__ perm, int n, ScanPack pk,
                          unsigned *__restrict__ status) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  uint32_t p = perm[j];
  if (p >= (uint32_t)n) {  // a sort defect: record it and keep the access in bounds
    atomicOr(status, 4u);
    p = (uint32_t)j;
  }
  // read-only loads; the gathered state is written with streaming stores (it
  // is read once, by the next propagation), the scan copies with plain ones
  const double x = __ldg(&src.x[p]), y = __ldg(&src.y[p]), z = __ldg(&src.z[p]);
  const double vx = __ldg(&src.vx[p]), vy = __ldg(&src.vy[p]), vz = __ldg(&src.vz[p]);
  const uint32_t tag = __ldg(&src.tag[p]);
  const double radius = tagSlot(tag) < (uint32_t)n ? __ldg(&src.radius[tagSlot(tag)]) : 0.0;  // slot-indexed
  if (pk.grp) pk.grp[j] = tagSlot(tag) < (uint32_t)n ? groupOf(src.parent[tagSlot(tag)]) : kNoGroup;
  __stcs(&dst.x[j], x);
  __stcs(&dst.y[j], y);
  __stcs(&dst.z[j], z);
  __stcs(&dst.vx[j], vx);
  __stcs(&dst.vy[j], vy);
  __stcs(&dst.vz[j], vz);
  __stcs(&dst.aom[j], __ldg(&src.aom[p]));
  __stcs(&dst.bc[j], __ldg(&src.bc[p]));
  __stcs(&dst.tag[j], tag);
  pk.posf[j] = floatPosition(x, y, z);
  pk.velf[j] = make_float4((float)vx, (float)vy, (float)vz, __double2float_ru(radius));
}

__device__ __forceinline__ double dot3rn(const double a[3], const double b[3]) {
  double r = __dadd_rn(0.0, __dmul_rn(a[0], b[0]));
  r = __dadd_rn(r, __dmul_rn(a[1], b[1]));
  return __dadd_rn(r, __dmul_rn(a[2], b[2]));
}

// distanceByLinearInterpolation (DistanceApproximation.cpp:13-58); returns the
// clamped closest-approach parameter t in [0, dt] (measured from r - v dt)
__device__ __forceinline__ double interpolate(const double ri[3], const double vi[3], const double rj[3],
                                            const double vj[3], double dt, double dr[3], double p2[3]) {
  double oi[3], oj[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    oi[k] = __dsub_rn(ri[k], __dmul_rn(vi[k], dt));
    oj[k] = __dsub_rn(rj[k], __dmul_rn(vj[k], dt));
  }
  const double vi_ri = dot3rn(vi, oi), vi_rj = dot3rn(vi, oj), vj_ri = dot3rn(vj, oi), vj_rj = dot3rn(vj, oj);
  const double num = __dsub_rn(__dsub_rn(__dadd_rn(vi_rj, vj_ri), vi_ri), vj_rj);
  const double two = __dmul_rn(2.0, dot3rn(vi, vj));
  const double den = __dsub_rn(__dadd_rn(dot3rn(vi, vi), dot3rn(vj, vj)), two);
  double t = __ddiv_rn(num, den);
  t = (t < 0.0) ? 0.0 : ((dt < t) ? dt : t);  // std::clamp: NaN passes
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double p1 = __dadd_rn(oi[k], __dmul_rn(vi[k], t));
    p2[k] = __dadd_rn(oj[k], __dmul_rn(vj[k], t));
    dr[k] = __dsub_rn(p1, p2[k]);
  }
  return t;
}

__device__ __forceinline__ bool nearBand(double x, double thr2, double rel) {
  return fabs(__dsub_rn(x, thr2)) <= __dmul_rn(rel, thr2);
}

struct Obj {
  double r[3], v[3], radius;
  uint64_t id, parent;
  uint32_t tag;
};

// (positions by the pre-gather position perm[k], radius / id / parent by slot)
__device__ __forceinline__ void loadObjPacked(const ScanPack &pk, uint32_t k, Obj &o) {
  const uint32_t p = pk.perm[k];
  o.r[0] = pk.src.x[p];
  o.r[1] = pk.src.y[p];
  o.r[2] = pk.src.z[p];
  o.v[0] = pk.src.vx[p];
  o.v[1] = pk.src.vy[p];
  o.v[2] = pk.src.vz[p];
  o.tag = pk.src.tag[p];
  const uint32_t s = tagSlot(o.tag);
  o.radius = pk.src.radius[s];
  o.id = pk.src.id[s];
  o.parent = pk.src.parent[s];
}

// CollisionFunctor::AoSFunctor on (i, j) with the gate already evaluated.
__device__ __forceinline__ uint32_t functorPair(const ScanConsts &c, const Obj &I, const Obj &J, double d2,
                                                double &dl2, double point[3]) {
  const int ai = tagAct(I.tag), aj = tagAct(J.tag);
  const bool wasEvaded = (ai != kPassive && aj != kPassive) || (ai != kPassive && J.radius >= c.minDetectionRadius) ||
                         (aj != kPassive && I.radius >= c.minDetectionRadius);
  if (I.parent != UINT64_MAX && I.parent == J.parent) return 0u;
  uint32_t flags = nearBand(d2, c.cutoffSq, c.nearRel) ? LADDS_PAIR_NEAR_GATE : 0u;
  const bool gate = !(d2 > c.cutoffSq);
  if (!gate && !flags) return 0u;
  double drl[3], p2[3];
  interpolate(I.r, I.v, J.r, J.v, c.dt, drl, p2);
  dl2 = dot3rn(drl, drl);
#pragma unroll
  for (int k = 0; k < 3; ++k) point[k] = __dadd_rn(p2[k], __dmul_rn(drl[k], 0.5));
  if (!gate) return flags;
  if (wasEvaded) {
    if (!(dl2 > c.evasionSq)) flags |= LADDS_PAIR_EVASION;
    if (nearBand(dl2, c.evasionSq, c.nearRel)) flags |= LADDS_PAIR_NEAR_EVASION;
  } else {
    const double sep = __dmul_rn(__dadd_rn(I.radius, J.radius), c.factor);
    const double sep2 = __dmul_rn(sep, sep);
    if (!(dl2 > sep2)) flags |= LADDS_PAIR_COLLISION;
    if (nearBand(dl2, sep2, c.nearRel)) flags |= LADDS_PAIR_NEAR_COLLISION;
  }
  if (!(dl2 > c.conjSq)) flags |= LADDS_PAIR_CONJUNCTION;
  if (nearBand(dl2, c.conjSq, c.nearRel)) flags |= LADDS_PAIR_NEAR_CONJUNCTION;
  return flags;
}

// Binary32 screen of a candidate pair: false only if the pair provably yields
// no record, i.e. its closest approach over the step exceeds every threshold
// (collision separation with the radii rounded up, evasion and conjunction
// cutoffs, their near bands) and d^2 is outside the near band of the cutoff,
// each by more than the error bound of this computation:
//   positions: per-coordinate rounding <= posf.w (a 4x bound), velocities
//   2^-24 |v| per coordinate, times dt; the closest approach over t is
//   1-Lipschitz in the separation and dt-Lipschitz in the relative velocity;
//   binary32 arithmetic on separations of size S: 2^-20 S.  FAST: the division
//   and the square roots are the hardware approximations (relative errors of
//   a few 2^-23): an error in t moves the distance at second order, and the
//   distances' own relative error stays far inside the 1e-6 S term.  (FAST
//   pays where the screen dominates -- dense populations -- and costs where it
//   does not: its special-function work competes with the propagation that
//   runs beside the scan.)
// NaN (identical velocities: the reference's 0/0 path) keeps the pair.
// the binary32 constants of mayRecord from the scan's parameters (host):
// dt, factor; rel = 1 + 4 nearRel + 1e-6; thr = max(evasion cutoff, conjunction
// threshold); cutoff^2, cutoff; nearBand = cutoff^2 nearRel 1.01.  Computed
// once per scan instead of per screened pair (each was a conversion from
// binary64 or a square root); the values are those the screen formed itself.
inline ScanConsts screenConsts(ScanConsts c) {
  c.dtF = (float)c.dt;
  c.factorF = (float)c.factor;
  const float nr = (float)c.nearRel;
  c.relF = 1.0f + 4.0f * nr + 1e-6f;
  c.thrF = std::max(std::sqrt((float)c.evasionSq), std::sqrt((float)c.conjSq));
  c.cut2F = (float)c.cutoffSq;
  c.cutF = std::sqrt(c.cut2F);
  c.nearBandF = c.cut2F * nr * 1.01f;
  return c;
}

template <bool FAST = false>
__device__ __forceinline__ bool mayRecord(const ScanConsts &c, float4 pa, float4 va, float4 pb, float4 vb) {
  const float dt = c.dtF;
  const float drx = pa.x - pb.x, dry = pa.y - pb.y, drz = pa.z - pb.z;
  const float dvx = va.x - vb.x, dvy = va.y - vb.y, dvz = va.z - vb.z;
  const float ox = drx - dvx * dt, oy = dry - dvy * dt, oz = drz - dvz * dt;  // separation at the step start
  const float dv2 = dvx * dvx + dvy * dvy + dvz * dvz;
  const float num = -(ox * dvx + oy * dvy + oz * dvz);
  float t = FAST ? __fdividef(num, dv2) : num / dv2;  // 0/0: NaN, kept below
  t = (t < 0.0f) ? 0.0f : ((dt < t) ? dt : t);
  const float mx = ox + dvx * t, my = oy + dvy * t, mz = oz + dvz * t;
  const float m2 = mx * mx + my * my + mz * mz;
  const float dl = FAST ? m2 * rsqrtf(m2) : sqrtf(m2);  // FAST: 0 * inf = NaN for m2 = 0, kept
  const float d2 = drx * drx + dry * dry + drz * drz;
  const float vmax = fmaxf(fmaxf(fabsf(va.x), fabsf(va.y)), fabsf(va.z)) +
                     fmaxf(fmaxf(fabsf(vb.x), fabsf(vb.y)), fabsf(vb.z));
  const float sepScale = FAST ? d2 * rsqrtf(d2) + dv2 * rsqrtf(dv2) * dt : sqrtf(d2) + sqrtf(dv2) * dt;
  const float err = 3.5f * (pa.w + pb.w) + 3.5e-7f * vmax * dt + 1e-6f * sepScale + 1e-6f;
  const float sep = (va.w + vb.w) * c.factorF;
  const float thr = fmaxf(sep, c.thrF) * c.relF;
  if (!(dl > thr + err)) return true;  // also NaN
  // near band of the cutoff gate: |d^2 - cutoff^2| <= nearRel cutoff^2
  const float d2err = 2.0f * c.cutF * err + 1e-5f * c.cut2F;
  return fabsf(d2 - c.cut2F) <= c.nearBandF + d2err;
}

__device__ __forceinline__ uint32_t lowerBound(const uint32_t *__restrict__ a, uint32_t lo, uint32_t hi, uint32_t v) {
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (a[mid] < v)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

__device__ __forceinline__ void emitPair(const Obj &I, const Obj &J, double dl2, const double point[3],
                                         uint32_t flags, uint32_t step, ladds_pair *__restrict__ out,
                                         unsigned long long *__restrict__ count, unsigned long long cap) {
  const unsigned long long pos = atomicAdd(count, 1ull);
  if (pos < cap) {
    ladds_pair p;
    p.idA = I.id;
    p.idB = J.id;
    p.slotA = tagSlot(I.tag);
    p.slotB = tagSlot(J.tag);
    p.dl2 = dl2;
    p.point[0] = point[0];
    p.point[1] = point[1];
    p.point[2] = point[2];
    p.step = step;
    p.flags = flags;
    out[pos] = p;
  }
}

// Scatter the sorted population back to slot order (download path).
// (slots are dense in [0, n); the guards only keep a corrupted tag in bounds)
__global__ void k_unpermute_f64(const double *__restrict__ src, const uint32_t *__restrict__ tag, int n,
                                double *__restrict__ dst) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n && tagSlot(tag[j]) < (uint32_t)n) dst[tagSlot(tag[j])] = src[j];
}
__global__ void k_unpermute_act(const uint32_t *__restrict__ tag, int n, int8_t *__restrict__ dst) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n && tagSlot(tag[j]) < (uint32_t)n) dst[tagSlot(tag[j])] = (int8_t)tagAct(tag[j]);
}
__global__ void k_unpermute_tag(const uint32_t *__restrict__ tag, int n, uint32_t *__restrict__ dst) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n && tagSlot(tag[j]) < (uint32_t)n) dst[tagSlot(tag[j])] = tag[j];
}
// Gather slot-ordered values into the current (sorted) order (state upload).
__global__ void k_permute_from_slots_f64(const double *__restrict__ src, const uint32_t *__restrict__ tag, int n,
                                         double *__restrict__ dst) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n && tagSlot(tag[j]) < (uint32_t)n) dst[j] = src[tagSlot(tag[j])];
}

__global__ void k_clear_parents(uint64_t *__restrict__ parent, int n) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n) parent[j] = UINT64_MAX;
}

// slotMark[slot] = 1 for slots to delete
__global__ void k_mark_deleted(uint32_t *__restrict__ tag, const uint8_t *__restrict__ slotMark, int n) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n && tagSlot(tag[j]) < (uint32_t)n && slotMark[tagSlot(tag[j])]) tag[j] |= kTagDummy;
}

// keep[j] = 1 if the object survives the burn-up test |r|^2 >= crit^2
// (Simulation.cpp:581-590); aliveBySlot[slot] mirrors it in slot order;
// *burnt counts the objects that fail it (one atomic per warp that has any).
__global__ void k_burnup_flags(const double *__restrict__ x, const double *__restrict__ y,
                               const double *__restrict__ z, const uint32_t *__restrict__ tag, int n,
                               double critSq, uint32_t *__restrict__ keep, uint32_t *__restrict__ aliveBySlot,
                               unsigned *__restrict__ burnt) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t k = 1u;
  if (j < n) {
    const double a2 = x[j] * x[j] + y[j] * y[j] + z[j] * z[j];
    k = (a2 < critSq) ? 0u : 1u;
    keep[j] = k;
    if (tagSlot(tag[j]) < (uint32_t)n) aliveBySlot[tagSlot(tag[j])] = k;
  }
  const unsigned below = __ballot_sync(0xffffffffu, k == 0u);
  if (below && (threadIdx.x & 31) == 0) atomicAdd(burnt, (unsigned)__popc(below));
}

// (slot, id) of every object with keep[j] == 0, appended in any order to
// outSlot / outIdLo / outIdHi (count[0] = their number): the ids of a removal
// go to the host without copying population-sized arrays.
__global__ void k_removed_ids(const uint32_t *__restrict__ keep, const uint32_t *__restrict__ tag,
                              const uint64_t *__restrict__ idBySlot, int n, uint32_t *__restrict__ outSlot,
                              uint32_t *__restrict__ outIdLo, uint32_t *__restrict__ outIdHi,
                              unsigned *__restrict__ count) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n || keep[j]) return;
  const uint32_t slot = tagSlot(tag[j]);
  const uint32_t q = atomicAdd(count, 1u);
  const uint64_t id = slot < (uint32_t)n ? idBySlot[slot] : 0ull;
  outSlot[q] = slot;
  outIdLo[q] = (uint32_t)id;
  outIdHi[q] = (uint32_t)(id >> 32);
}

// keep[j] = 0 for the objects that leave the container: a position or
// velocity that is not finite, or a position outside [boxMin, boxMax]
// (AutoPas::updateContainer's leaving particles, Simulation.cpp:314; a NaN
// position is inside no box); aliveBySlot mirrors keep in slot order.
__global__ void k_escape_flags(DevState s, int n, double3 lo, double3 hi, uint32_t *__restrict__ keep,
                               uint32_t *__restrict__ aliveBySlot, unsigned *__restrict__ escaped) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t k = 1u;
  if (j < n) {
    const double x = s.x[j], y = s.y[j], z = s.z[j];
    const bool inside = x >= lo.x && x <= hi.x && y >= lo.y && y <= hi.y && z >= lo.z && z <= hi.z;
    const bool finiteV = isfinite(s.vx[j]) && isfinite(s.vy[j]) && isfinite(s.vz[j]);
    k = (inside && finiteV) ? 1u : 0u;
    keep[j] = k;
    if (tagSlot(s.tag[j]) < (uint32_t)n) aliveBySlot[tagSlot(s.tag[j])] = k;
  }
  const unsigned out = __ballot_sync(0xffffffffu, k == 0u);
  if (out && (threadIdx.x & 31) == 0) atomicAdd(escaped, (unsigned)__popc(out));
}

// keep[j] = 0 for the objects whose slot is marked (slotMark[slot] = 1);
// aliveBySlot mirrors it in slot order.
__global__ void k_slot_mark_flags(const uint32_t *__restrict__ tag, int n, const uint8_t *__restrict__ slotMark,
                                  uint32_t *__restrict__ keep, uint32_t *__restrict__ aliveBySlot) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const uint32_t s = tagSlot(tag[j]);
  const uint32_t k = (s < (uint32_t)n && slotMark[s]) ? 0u : 1u;
  keep[j] = k;
  if (s < (uint32_t)n) aliveBySlot[s] = k;
}

// compaction: dst[pos[j]] = src[j] for kept j, slots renumbered via newSlot;
// the slot-indexed arrays go to the new slots of separate arrays (tRadius,
// tId, tParent), as the state buffers share theirs
__global__ void k_compact(DevState src, DevState dst, const uint32_t *__restrict__ keep,
                          const uint32_t *__restrict__ pos, const uint32_t *__restrict__ newSlot, int n,
                          double *__restrict__ tRadius, uint64_t *__restrict__ tId, uint64_t *__restrict__ tParent) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n || !keep[j]) return;
  const uint32_t p = pos[j];
  dst.x[p] = src.x[j];
  dst.y[p] = src.y[j];
  dst.z[p] = src.z[j];
  dst.vx[p] = src.vx[j];
  dst.vy[p] = src.vy[j];
  dst.vz[p] = src.vz[j];
  dst.aom[p] = src.aom[j];
  dst.bc[p] = src.bc[j];
  const uint32_t t = src.tag[j], s = tagSlot(t);
  if (s >= (uint32_t)n) return;  // only with a corrupted tag
  const uint32_t ns = newSlot[s];
  dst.tag[p] = (t & ~kTagSlotMask) | (ns & kTagSlotMask);
  tRadius[ns] = src.radius[s];
  tId[ns] = src.id[s];
  tParent[ns] = src.parent[s];
}

// exclusive scan of u32 flags, three phases (block sums, scan of sums, apply)
constexpr int kScanBlock = 1024;
__global__ void __launch_bounds__(kScanBlock) k_scan_blocks(const uint32_t *__restrict__ in, int n,
                                                            uint32_t *__restrict__ out,
                                                            uint32_t *__restrict__ blockSums) {
  __shared__ uint32_t ws[32];
  const int i = blockIdx.x * kScanBlock + threadIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t v = i < n ? in[i] : 0u;
  uint32_t incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) ws[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = ws[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += t;
    }
    ws[lane] = w;
  }
  __syncthreads();
  const uint32_t off = warp ? ws[warp - 1] : 0u;
  if (i < n) out[i] = off + incl - v;
  if (threadIdx.x == kScanBlock - 1) blockSums[blockIdx.x] = off + incl;
}

// second pass of a two-pass exclusive scan (at most kScanBlock blocks): block b
// adds the sum of blockSums[0, b) -- the scan of the block sums folded into
// the apply pass
__global__ void __launch_bounds__(kScanBlock) k_scan_add_prefix(uint32_t *__restrict__ out, int n,
                                                                const uint32_t *__restrict__ blockSums) {
  __shared__ uint32_t ws[32];
  const int b = blockIdx.x, t = threadIdx.x;
  const uint32_t w = __reduce_add_sync(0xffffffffu, t < b ? blockSums[t] : 0u);
  if ((t & 31) == 0) ws[t >> 5] = w;
  __syncthreads();
  const uint32_t off = __reduce_add_sync(0xffffffffu, ws[t & 31]);  // every warp sums the 32 partials
  const int i = b * kScanBlock + t;
  if (i < n && b > 0) out[i] += off;
}

__global__ void k_scan_add(uint32_t *__restrict__ out, int n, const uint32_t *__restrict__ blockOffsets) {
  const int i = blockIdx.x * kScanBlock + threadIdx.x;
  if (i < n) out[i] += blockOffsets[blockIdx.x];
}

}  // namespace ladds
