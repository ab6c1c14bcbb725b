// Integrator.h -- drop-in for YoshidaIntegrator<AutoPas_t> (constructed at
// src/ladds/Simulation.cpp:122-148, integrate(false) called at :297).
//
// The acceleration components are the reference's std::array<bool, 8> mask
// (KEP, J2, C22, S22, SOL, LUN, SRP, DRAG; Simulation.cpp:127-135) plus J3.
// integrate() runs one Yoshida-4 step of every particle on the GPU.  In the
// host-owned mode (default) the container is uploaded when it changed (another
// container, or another size; after changing particles in place at the same
// size call GpuContext::invalidate()) and the new positions / velocities are
// written back after every step, as the reference integrator updates the
// particles in place; in the device-resident mode the state stays on the GPU
// until sync().
#pragma once
#include <array>

#include "ladds/GpuContext.h"

namespace ladds {

class Integrator {
 public:
  Integrator(Container &container, GpuContext &gpu) : container_(container), gpu_(gpu) {}

  // One step (outputToFile is accepted for call compatibility; the propagator's
  // CSV output is not part of the hot path).
  void integrate(bool outputToFile = false);
  // Several steps in one device call (one launch per 128 steps).
  void integrate(int steps);
  void setDeviceResident(bool resident) { resident_ = resident; }
  // device -> container (device-resident mode)
  void sync() { gpu_.downloadState(container_); }

  static uint32_t componentMask(const std::array<bool, 8> &components, bool useJ3);

 private:
  void ensureUploaded();
  Container &container_;
  GpuContext &gpu_;
  bool resident_ = false;
};

}  // namespace ladds
