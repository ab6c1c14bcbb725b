// GpuCollisionFunctor.h -- the CollisionFunctor contract on the GPU.
//
// Same construction and results as the reference's CollisionFunctor
// (src/ladds/CollisionFunctor.h:22-129, .cpp:18-246):
//   GpuCollisionFunctor(cutoff, dt, collisionDistanceFactor, minDetectionRadius,
//                       evasionTrackingCutoffInKM)
//   initTraversal(); AoSFunctor(i, j, newton3) ...; endTraversal(newton3);
//   getCollisions(); getEvadedCollisions();
// AoSFunctor calls are queued and evaluated together on the GPU in
// endTraversal (ladds_gpu_functor_pairs).  run(container) replaces
// AutoPas::iteratePairwise(&functor) (Simulation.cpp:220): the whole
// linked-cell traversal runs on the GPU (ladds_gpu_scan).  Pairs are (lower id,
// higher id) as in CollisionFunctor.cpp:96-129 and the lists come out sorted by
// (idA, idB) -- the reference's order is that of its OpenMP thread buffers.
// Besides the two reference lists, getConjunctions() holds every gated pair
// closer than conjunctionThresholdInKM and getNearThreshold() the pairs within
// the near band of one of the thresholds.
#pragma once
#include <array>
#include <tuple>
#include <utility>
#include <vector>

#include "ladds/GpuContext.h"

namespace ladds {

class GpuCollisionFunctor {
 public:
  using CollisionT = std::tuple<Particle *, Particle *, double, std::array<double, 3>>;
  using CollisionCollectionT = std::vector<CollisionT>;

  GpuCollisionFunctor(double cutoff, double dt, double collisionDistanceFactor, double minDetectionRadius,
                      double evasionTrackingCutoffInKM, GpuContext &gpu, double conjunctionThresholdInKM = 0.1);

  bool allowsNewton3() const { return true; }
  bool allowsNonNewton3() const { return false; }  // CollisionFunctor.h:47-50
  bool isRelevantForTuning() const { return true; }

  void initTraversal();
  void AoSFunctor(Particle &i, Particle &j, bool newton3);
  void endTraversal(bool newton3);
  // iteratePairwise replacement over the whole container
  void run(Container &container, size_t iteration = 0);

  const CollisionCollectionT &getCollisions() const { return collisions_; }
  const CollisionCollectionT &getEvadedCollisions() const { return evasions_; }
  const CollisionCollectionT &getConjunctions() const { return conjunctions_; }
  const CollisionCollectionT &getNearThreshold() const { return near_; }
  const std::vector<ladds_pair> &records() const { return records_; }

 private:
  void distribute(const std::vector<ladds_pair> &recs, Particle *const *bySlot);
  ladds_scan_params params_;
  GpuContext &gpu_;
  std::vector<std::pair<Particle *, Particle *>> queue_;
  CollisionCollectionT collisions_, evasions_, conjunctions_, near_;
  std::vector<ladds_pair> records_;
};

}  // namespace ladds
