// insert.cuh -- checked insertion of new satellites (Simulation::checkedInsert,
// Simulation.cpp:475-507).
//
// A new satellite at p is inserted only if no particle q inside the box
// [p - c, p + c) (the AutoPas region iterator's half-open box, corners from
// ArrayMath::sub / add) has dot(p - q, p - q) <= c^2 (collisionFree =
// dot > c^2, so NaN also blocks); c = io/constellationCutoff.  The kernel tests
// every new satellite against the device population (deleted objects are
// absent in the reference and skipped here); satellites of the same batch are
// tested against the ones accepted before them on the host, in batch order.
#pragma once
#include "conjunction.cuh"
#include "propagate.cuh"

namespace ladds {

// the reference's test of one particle q against a satellite at p
__host__ __device__ __forceinline__ bool insertBlocks(const double p[3], const double q[3], double c, double c2) {
#ifdef __CUDA_ARCH__
#define LADDS_ADD(a, b) __dadd_rn(a, b)
#define LADDS_SUB(a, b) __dsub_rn(a, b)
#define LADDS_MUL(a, b) __dmul_rn(a, b)
#else
#define LADDS_ADD(a, b) ((a) + (b))
#define LADDS_SUB(a, b) ((a) - (b))
#define LADDS_MUL(a, b) ((a) * (b))
#endif
  for (int k = 0; k < 3; ++k) {
    const double lo = LADDS_SUB(p[k], c), hi = LADDS_ADD(p[k], c);
    if (!(q[k] >= lo && q[k] < hi)) return false;  // outside the region iterator's box
  }
  const double d0 = LADDS_SUB(p[0], q[0]), d1 = LADDS_SUB(p[1], q[1]), d2 = LADDS_SUB(p[2], q[2]);
  double s = LADDS_ADD(0.0, LADDS_MUL(d0, d0));
  s = LADDS_ADD(s, LADDS_MUL(d1, d1));
  s = LADDS_ADD(s, LADDS_MUL(d2, d2));
#undef LADDS_ADD
#undef LADDS_SUB
#undef LADDS_MUL
  return !(s > c2);
}

// one warp per new satellite: blocked[i] = some live particle of the state blocks it
__global__ void k_insert_blocked(DevState s, int n, const double *__restrict__ nx, const double *__restrict__ ny,
                                 const double *__restrict__ nz, int nNew, double c, double c2,
                                 uint8_t *__restrict__ blocked) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= nNew) return;  // whole warps exit together
  const double p[3] = {nx[w], ny[w], nz[w]};
  bool hit = false;
  for (int jb = 0; jb < n; jb += 32) {  // warp-uniform trip count
    const int j = jb + lane;
    if (j < n && !tagDummy(s.tag[j])) {
      const double q[3] = {s.x[j], s.y[j], s.z[j]};
      hit = hit || insertBlocks(p, q, c, c2);
    }
    if (__any_sync(0xffffffffu, hit)) break;
  }
  hit = __any_sync(0xffffffffu, hit);
  if (lane == 0) blocked[w] = hit ? 1 : 0;
}

// pos[q] = position in the state arrays of wanted slot q (wanted sorted ascending)
__global__ void k_find_slots(const uint32_t *__restrict__ tags, int n, const uint32_t *__restrict__ wanted, int m,
                             int32_t *__restrict__ pos) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const uint32_t slot = tagSlot(tags[j]);
  int lo = 0, hi = m;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (wanted[mid] < slot)
      lo = mid + 1;
    else
      hi = mid;
  }
  if (lo < m && wanted[lo] == slot) pos[lo] = j;
}

__global__ void k_gather_records(DevState s, const int32_t *__restrict__ pos, int m,
                                 ladds_state_record *__restrict__ out) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= m) return;
  const int32_t j = pos[q];
  if (j < 0) return;
  ladds_state_record r;
  r.r[0] = s.x[j];
  r.r[1] = s.y[j];
  r.r[2] = s.z[j];
  r.v[0] = s.vx[j];
  r.v[1] = s.vy[j];
  r.v[2] = s.vz[j];
  const uint32_t slot = tagSlot(s.tag[j]);  // radius, id and parent are indexed by slot
  r.radius = s.radius[slot];
  r.aom = s.aom[j];
  r.bcInv = s.bc[j];
  r.id = s.id[slot];
  r.parentId = s.parent[slot];
  r.activity = tagAct(s.tag[j]);
  r.deleted = tagDummy(s.tag[j]) ? 1u : 0u;
  out[q] = r;
}

// Layer selection of the device-resident exchange (ladds_gpu_pack_layers):
// sel[j] = 1 for the live objects whose cell layer lies in [lo, hi), keep[j]
// = !sel[j] and aliveBySlot its slot-order mirror (for the removal).
__global__ void k_layer_flags(const double *__restrict__ z, const uint32_t *__restrict__ tag, int n, GridDesc g,
                              int32_t lo, int32_t hi, uint32_t *__restrict__ sel, uint32_t *__restrict__ keep,
                              uint32_t *__restrict__ aliveBySlot) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const uint32_t t = tag[j];
  const int32_t iz = (int32_t)cellCoord(z[j], g.boxMin[2], g.invCell, g.n[2]);
  const uint32_t s = (!tagDummy(t) && iz >= lo && iz < hi) ? 1u : 0u;
  sel[j] = s;
  keep[j] = 1u - s;
  if (tagSlot(t) < (uint32_t)n) aliveBySlot[tagSlot(t)] = 1u - s;
}

// positions of the selected objects in their (current) order: idx[pos[j]] = j
__global__ void k_selected_positions(const uint32_t *__restrict__ sel, const uint32_t *__restrict__ pos, int n,
                                     int32_t *__restrict__ idx) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n && sel[j]) idx[pos[j]] = j;
}

// State records (device memory) appended at positions / slots offset..offset+m
// (slot-indexed radius, id and parent at the same index); bad[0] counts
// records with a non-finite value or an activity state out of range, bad[1]
// is set when a record has a parent id.
__global__ void k_append_records(const ladds_state_record *__restrict__ in, int m, DevState s, uint32_t offset,
                                 unsigned *__restrict__ bad) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= m) return;
  const ladds_state_record r = in[q];
  const uint32_t at = offset + (uint32_t)q;
  const bool ok = isfinite(r.r[0]) && isfinite(r.r[1]) && isfinite(r.r[2]) && isfinite(r.v[0]) &&
                  isfinite(r.v[1]) && isfinite(r.v[2]) && isfinite(r.radius) && isfinite(r.aom) &&
                  isfinite(r.bcInv) && r.activity >= 0 && r.activity <= 2;
  if (!ok) atomicAdd(bad, 1u);
  if (r.parentId != UINT64_MAX) atomicOr(bad + 1, 1u);
  s.x[at] = r.r[0];
  s.y[at] = r.r[1];
  s.z[at] = r.r[2];
  s.vx[at] = r.v[0];
  s.vy[at] = r.v[1];
  s.vz[at] = r.v[2];
  s.aom[at] = r.aom;
  s.bc[at] = r.bcInv;
  s.radius[at] = r.radius;
  s.id[at] = r.id;
  s.parent[at] = r.parentId;
  s.tag[at] = makeTag(at, ok ? r.activity : 0, r.deleted != 0u);
}

// keep[j] = slot < n0 (the removal of a truncation), aliveBySlot its mirror
__global__ void k_truncate_flags(const uint32_t *__restrict__ tag, int n, uint32_t n0, uint32_t *__restrict__ keep,
                                 uint32_t *__restrict__ aliveBySlot) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const uint32_t sl = tagSlot(tag[j]);
  const uint32_t k = sl < n0 ? 1u : 0u;
  keep[j] = k;
  if (sl < (uint32_t)n) aliveBySlot[sl] = k;
}

}  // namespace ladds
