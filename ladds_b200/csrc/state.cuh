// state.cuh -- device layout of the particle population.
//
// Structure of arrays, one array per attribute of the reference Particle
// (Particle.h:139-195) that the hot path reads.  Positions and velocities are
// binary64 (48 B/object), the per-object constants aom / bcInv / radius are
// binary64, id / parentId are u64 and a u32 tag packs the slot (upload index),
// the activity state and the dummy ("deleted") flag.  Two copies are kept and
// swapped: every conjunction scan gathers the population into cell order, so
// objects stay spatially sorted and the next gather is close to a streaming copy.
#pragma once
#include <cstdint>

namespace ladds {

constexpr uint32_t kTagSlotBits = 28;
constexpr uint32_t kTagSlotMask = (1u << kTagSlotBits) - 1u;
constexpr uint32_t kTagActShift = 28;
constexpr uint32_t kTagDummy = 1u << 31;
constexpr size_t kMaxObjects = (size_t)kTagSlotMask;  // 268 M

__host__ __device__ __forceinline__ uint32_t makeTag(uint32_t slot, int act, bool dummy) {
  return (slot & kTagSlotMask) | ((uint32_t)(act & 3) << kTagActShift) | (dummy ? kTagDummy : 0u);
}
__host__ __device__ __forceinline__ uint32_t tagSlot(uint32_t t) { return t & kTagSlotMask; }
__host__ __device__ __forceinline__ int tagAct(uint32_t t) { return (int)((t >> kTagActShift) & 3u); }
__host__ __device__ __forceinline__ bool tagDummy(uint32_t t) { return (t & kTagDummy) != 0; }

// One state buffer.  x .. vz, aom, bc and tag are indexed by position (the
// order the buffer holds the objects in); radius, id and parent are indexed by
// slot (tagSlot of the tag), do not move when the population is gathered into
// cell order, and are shared by a context's buffers.
struct DevState {
  double *x, *y, *z, *vx, *vy, *vz;
  double *aom, *bc, *radius;
  uint64_t *id, *parent;
  uint32_t *tag;
};

// cell grid: key = (iz * ny + iy) * nx + ix
struct GridDesc {
  double boxMin[3];
  double cellSize, invCell;
  int32_t n[3];
  int32_t reach;
  uint32_t keyBits;
};

struct ScanConsts {
  double cutoffSq;    // cutoff * cutoff                        (CollisionFunctor.cpp:24)
  double dt;          // interpolation window
  double factor;      // collisionDistanceFactor / 1000.        (CollisionFunctor.cpp:26)
  double minDetectionRadius;
  double evasionSq;   // evasionCutoff * evasionCutoff          (CollisionFunctor.cpp:28)
  double conjSq;      // conjunctionThreshold^2
  double nearRel;
  // binary32 forms for the screen of the pair scan (mayRecord), derived from the
  // fields above by screenConsts() before every scan launch
  float dtF, factorF, relF, thrF, cut2F, cutF, nearBandF;
};

}  // namespace ladds
