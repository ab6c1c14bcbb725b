// HotPathLoop.h -- the hot-path part of Simulation::simulationLoop
// (src/ladds/Simulation.cpp:287-415) on the GPU:
//   - after 100 iterations without a collision every parent id is reset
//     (spawn protection, :291-293, :470-473);
//   - integrate one step (:297);
//   - delete burn-ups below minAltitude (:302, :561-596) and particles that
//     leave the container: outside the box or with a non-finite state (:314,
//     :381-387);
//   - every timestepsPerCollisionDetection iterations, the conjunction scan with
//     dt = deltaT * k (:389-397), collisions / evasions handed to the writer.
// The population stays on the device; the container is kept in step for
// burn-ups (erased by id) and written back by sync().
#pragma once
#include <functional>

#include "ladds/GpuCollisionFunctor.h"
#include "ladds/Integrator.h"

namespace ladds {

class HotPathLoop {
 public:
  using Writer = std::function<void(size_t iteration, const GpuCollisionFunctor::CollisionCollectionT &)>;

  HotPathLoop(ConfigReader &config, Container &container, GpuContext &gpu);
  // Runs iterations [first, first + n); returns the number of collisions
  // (Simulation::simulationLoop's "total conjunctions").
  size_t run(size_t n);
  void sync() { gpu_.downloadState(container_); }
  void setCollisionWriter(Writer w) { writeCollisions_ = std::move(w); }
  void setEvasionWriter(Writer w) { writeEvasions_ = std::move(w); }
  size_t totalEvasions() const { return totalEvasions_; }
  size_t escaped() const { return escaped_; }
  size_t iteration() const { return iteration_; }

 private:
  Container &container_;
  GpuContext &gpu_;
  double deltaT_, minAltitude_, cutoff_, factor_, minDetectionRadius_, evasionCutoff_, conjunctionThreshold_;
  size_t k_;
  std::vector<uint64_t> removedIds_;  // ids of the iteration's burn-ups (kept between iterations)
  size_t iteration_ = 0, iterationsSinceLastCollision_ = 0, totalEvasions_ = 0, escaped_ = 0;
  Writer writeCollisions_, writeEvasions_;
};

}  // namespace ladds
