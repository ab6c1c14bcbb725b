// Particle.h -- host-side debris object with the attribute set of the
// reference's LADDS::Particle (src/ladds/particle/Particle.h:21-195): FP64
// position / velocity, id, COSPAR identifier, activity state, mass, radius,
// area over mass, inverse ballistic coefficient, parent id (spawn protection)
// and the dummy ("deleted") ownership state.  The device holds the same
// attributes as structure-of-arrays; this class is the container element the
// drop-in keeps on the host.
#pragma once
#include <array>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <limits>
#include <string>

namespace ladds {

class Particle {
 public:
  // Particle.h:37-53
  enum class ActivityState : int { passive = 0, evasive = 1, evasivePreserving = 2 };

  // Inverse ballistic coefficient [m^2/kg] from B* when it is set, else from the
  // drag coefficient and the cross-section (Particle.cpp:13-27).
  static double calculateBcInv(double bstar, double mass, double radius, double coefficientOfDrag);

  // Particle.h:62-85; aom = pi r^2 1e-6 / m [km^2/kg]
  Particle(std::array<double, 3> pos, std::array<double, 3> v, size_t debrisId, std::string identifier,
           ActivityState activityState, double mass, double radius, double bcInv, size_t parentIdentifier);

  const std::array<double, 3> &getR() const { return r_; }
  const std::array<double, 3> &getPosition() const { return r_; }
  const std::array<double, 3> &getV() const { return v_; }
  const std::array<double, 3> &getVelocity() const { return v_; }
  void setR(const std::array<double, 3> &r) { r_ = r; }
  void setPosition(const std::array<double, 3> &r) { r_ = r; }
  void setV(const std::array<double, 3> &v) { v_ = v; }
  void setVelocity(const std::array<double, 3> &v) { v_ = v; }
  size_t getID() const { return id_; }
  void setID(size_t id) { id_ = id; }
  const std::string &getIdentifier() const { return identifier_; }
  ActivityState getActivityState() const { return activity_; }
  void setActivityState(ActivityState a) { activity_ = a; }
  double getMass() const { return mass_; }
  double getRadius() const { return radius_; }
  double getAom() const { return aom_; }
  double getBcInv() const { return bcInv_; }
  size_t getParentIdentifier() const { return parent_; }
  void setParentIdentifier(size_t p) { parent_ = p; }
  bool isDummy() const { return dummy_; }
  void setDummy(bool d) { dummy_ = d; }
  double getHeight() const { return std::sqrt(r_[0] * r_[0] + r_[1] * r_[1] + r_[2] * r_[2]); }
  double getSpeed() const { return std::sqrt(v_[0] * v_[0] + v_[1] * v_[1] + v_[2] * v_[2]); }

 private:
  std::array<double, 3> r_{}, v_{};
  size_t id_ = 0;
  std::string identifier_;
  ActivityState activity_ = ActivityState::passive;
  double mass_ = 0, radius_ = 0, aom_ = 0, bcInv_ = 0;
  size_t parent_ = std::numeric_limits<size_t>::max();
  bool dummy_ = false;
};

}  // namespace ladds
