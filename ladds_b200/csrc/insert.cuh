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

}  // namespace ladds
