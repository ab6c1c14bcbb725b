// GpuContext.h -- RAII owner of one ladds_gpu_ctx (include/ladds_gpu.h) and the
// host container of the drop-in.
//
// Container: the particle storage the host keeps (the reference keeps it in
// the AutoPas container, TypeDefinitions.h:13).  A std::deque keeps Particle*
// stable while particles are appended, so conjunction records can hold
// pointers into it as the reference's CollisionCollectionT does
// (CollisionFunctor.h:73-74).  Container index == device slot.
//
// Every non-zero status of the C ABI becomes a std::runtime_error carrying the
// library's message, as the reference reports errors
// (e.g. CollisionFunctor.cpp:186, Simulation.cpp:533).
#pragma once
#include <array>
#include <cstdint>
#include <deque>
#include <stdexcept>
#include <string>
#include <vector>

#include "ladds/ConfigReader.h"
#include "ladds/Particle.h"
#include "ladds_gpu.h"

namespace ladds {

using Container = std::deque<Particle>;

// Julian date of 00:00 UTC of a "yyyy-mm-dd" (or yyyy/mm/dd) calendar date.
double julianDate(const std::string &date);

class GpuContext {
 public:
  explicit GpuContext(const ladds_gpu_config &cfg);
  // Reads the keys of the hot path (sim/deltaT, sim/prop/use*Component,
  // sim/referenceTime, sim/maxAltitude, sim/collisionDistanceFactor,
  // sim/minDetectionRadius, sim/evasionTrackingCutoffInKM,
  // sim/conjunctionThresholdInKM, sim/timestepsPerCollisionDetection,
  // autopas/cutoff, gpu/{precision,cellSize,useGraphs,device}) with the
  // reference's defaults (Simulation.cpp:59-148, :233-247).
  static ladds_gpu_config configFrom(ConfigReader &config);
  ~GpuContext();
  GpuContext(const GpuContext &) = delete;
  GpuContext &operator=(const GpuContext &) = delete;

  ladds_gpu_ctx *handle() const { return ctx_; }
  const ladds_gpu_config &config() const { return cfg_; }
  void check(int status) const;

  // full upload of the container (dummies are marked deleted on the device)
  void upload(const Container &container);
  // positions / velocities of the device state written back into the container
  void downloadState(Container &container) const;
  // host <- device of every attribute (ids, parents, ...)
  void downloadAll(Container &container) const;
  size_t deviceSize() const;
  // the container last uploaded (pointer + size), to detect host-side changes
  bool mirrors(const Container &container) const;
  void markMirrored(const Container &container);
  // forgets the mirror, so that the next call uploads the container again:
  // needed after particles were changed in place with the size unchanged
  // (e.g. two removed and two appended), which the pointer + size test misses
  void invalidate() {
    mirror_ = nullptr;
    mirrorSize_ = 0;
  }

 private:
  ladds_gpu_config cfg_;
  ladds_gpu_ctx *ctx_ = nullptr;
  const Container *mirror_ = nullptr;
  size_t mirrorSize_ = 0;
};

}  // namespace ladds
